"""GPU parity: every stage of the CUDA SSAFD path against the CPU oracle, through the C-ABI.

Tolerances: FP64 stage values agree to 1e-12 relative (the GPU multiplies by
reciprocals of dx^2, dy^2, 2 dx dy, 4 dx dy and contracts to FMA where the oracle
divides); converged velocities agree to the parity bar of 1e-8 relative L2
with tight Picard / KSP tolerances.
"""
import numpy as np
import pytest

from pism_b200 import verification as V, synthetic as S
from pism_b200.config import SSAConfig, GridDesc, X_PERIODIC, Y_PERIODIC
from oracle import ssafd_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200.ssa import SSAFD, ZeroDiagonal  # noqa: E402

FIELDS = ("thickness", "surface", "bed", "mask", "tauc", "melange", "gl_mask", "enthalpy", "fracture_density")


def make_solver(g, c, f):
    s = SSAFD(g, c)
    kw = {k: f[k] for k in FIELDS if f.get(k) is not None}
    s.set_inputs(**kw, bc_mask=f.get("bc_mask"), bc_values=f.get("bc_values"))
    return s


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def random_case(seed, Mx=23, My=19, cfbc=False, dirichlet_bc=False, bc=True, periodicity=0, pseudo=False,
                sub_gl=False, eta=False, flow_law="isothermal_glen", nu_bedrock=False):
    """Random inputs exercising every mask configuration of a 3x3 neighbourhood."""
    rng = np.random.default_rng(seed)
    g = GridDesc(Mx, My, 0.5 * (Mx - 1) * 7e3, 0.5 * (My - 1) * 9e3, periodicity=periodicity,
                 z=np.linspace(0, 4000, 11))
    c = SSAConfig(calving_front_stress_boundary_condition=cfbc, ssa_dirichlet_bc=dirichlet_bc,
                  do_pseudo_plastic_till=pseudo, sub_groundingline=sub_gl,
                  surface_gradient_method="eta" if eta else "haseloff", flow_law=flow_law,
                  nu_bedrock_set=nu_bedrock)
    mask = rng.choice([0.0, 2.0, 3.0, 4.0], size=(Mx, My)) + rng.uniform(-0.3, 0.3, (Mx, My))
    Mi = np.floor(mask + 0.5)
    H = np.where((Mi == 2) | (Mi == 3), rng.uniform(20, 3000, (Mx, My)), rng.uniform(0, 30, (Mx, My)))
    H[rng.random((Mx, My)) < 0.05] = 0.0
    bed = rng.uniform(-1500, 1500, (Mx, My))
    f = {
        "thickness": H, "bed": bed, "surface": bed + H + rng.uniform(-5, 5, (Mx, My)), "mask": mask,
        "tauc": rng.uniform(1e3, 2e5, (Mx, My)), "melange": rng.uniform(0, 0.5, (Mx, My)),
        "gl_mask": rng.uniform(0, 1, (Mx, My)) if sub_gl else None,
        "enthalpy": rng.uniform(1.0e5, 2.0e5, (Mx, My, 11)) if flow_law != "isothermal_glen" else None,
    }
    if bc:
        bm = (rng.random((Mx, My)) < 0.1).astype(float)
        f["bc_mask"] = bm
        f["bc_values"] = rng.normal(0, 1e-5, (Mx, My, 2))
    return g, c, f


CASES = {
    "plain": dict(),
    "cfbc": dict(cfbc=True),
    "cfbc_dirichlet": dict(cfbc=True, dirichlet_bc=True),
    "no_bc": dict(bc=False),
    "pseudo_subgl": dict(pseudo=True, sub_gl=True),
    "eta": dict(eta=True),
    "xperiodic": dict(periodicity=X_PERIODIC),
    "yperiodic_inward": dict(periodicity=Y_PERIODIC),
    "nu_bedrock": dict(nu_bedrock=True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_stage_parity(name):
    g, c, f = random_case(sum(map(ord, name)), **CASES[name])
    if name == "yperiodic_inward":
        c.compute_surf_grad_inward_ssa = True
    G, Cc, I = O.from_case(g, c, f)
    s = make_solver(g, c, f)
    s.assemble_rhs()
    s.compute_hardav_staggered()
    taud = O.driving_stress(G, Cc, I)
    np.testing.assert_allclose(s.driving_stress(), taud, rtol=1e-12, atol=1e-9 * np.abs(taud).max())
    b = O.assemble_rhs(G, Cc, I, taud)
    np.testing.assert_allclose(s.rhs(), b, rtol=1e-12, atol=1e-9 * np.abs(b).max())
    hard = O.hardness_staggered(G, Cc, I)
    np.testing.assert_allclose(s.hardness(), hard, rtol=1e-12)
    rng = np.random.default_rng(1)
    vel = rng.normal(0, 3e-6, (g.Mx, g.My, 2))
    s.set_initial_guess(vel)
    s.compute_nuH_staggered(1e13)
    nuH = O.compute_nuH(G, Cc, I, hard, vel, 1e13)
    np.testing.assert_allclose(s.nuH(), nuH, rtol=1e-12)
    beta = O.beta_field(Cc, I, vel)
    np.testing.assert_allclose(s.beta(), beta, rtol=1e-12)
    # operator: GPU matrix-free apply vs the assembled 18-column matrix
    x = rng.normal(0, 1e-5, (g.Mx, g.My, 2))
    A = O.assemble_matrix(G, Cc, I, s.nuH(), s.beta(), check_diagonal=False)
    y_ref = (A @ x.ravel()).reshape(x.shape)
    xd = torch.tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    s.apply(xd, yd)
    torch.cuda.synchronize()
    y = yd.cpu().numpy()
    scale = (abs(A) @ np.abs(x).ravel()).reshape(x.shape)      # sum_m |a_m x_m| per row
    assert np.all(np.abs(y - y_ref) <= 1e-12 * scale + 1e-300), np.max(np.abs(y - y_ref) / (scale + 1e-300))
    s.close()


@pytest.mark.parametrize("pc,shape,periodicity", [("bjacobi", (23, 19), 0), ("line", (23, 19), 0),
                                                  ("line", (23, 19), Y_PERIODIC), ("line", (5, 601), 0),
                                                  ("line", (7, 512), X_PERIODIC)])
def test_preconditioner_apply_matches_oracle(pc, shape, periodicity):
    """z = M^-1 r (PCApply) against the oracle: block Jacobi inverts each cell's 2 x 2
    diagonal block; the line preconditioner solves the 2 x 2-block tridiagonal part of every
    grid line of constant i (no wrap across its ends), in chunks of 256 cells (601 = two
    full chunks and a partial one, 512 = exactly two).  Every mask case, Dirichlet rows
    included."""
    g, c, f = random_case(11 + shape[1], Mx=shape[0], My=shape[1], periodicity=periodicity)
    c.pc_type = pc
    G, Cc, I = O.from_case(g, c, f)
    s = make_solver(g, c, f)
    s.assemble_rhs()
    s.compute_hardav_staggered()
    rng = np.random.default_rng(2)
    s.set_initial_guess(rng.normal(0, 3e-6, (g.Mx, g.My, 2)))
    s.compute_nuH_staggered(1e13)
    A = O.assemble_matrix(G, Cc, I, s.nuH(), s.beta(), check_diagonal=False)
    if pc == "line":
        M = O.line_block_part(G, A)
    else:
        A = A.tocoo()
        keep = A.row // 2 == A.col // 2
        M = O.sp.csr_matrix((A.data[keep], (A.row[keep], A.col[keep])), shape=A.shape)
    r = rng.standard_normal((g.Mx, g.My, 2))
    rd = torch.tensor(r, device="cuda")
    zd = torch.empty_like(rd)
    s.apply_preconditioner(rd, zd)
    torch.cuda.synchronize()
    z = zd.cpu().numpy()
    # backward error of the device solve, row by row: |r - M z| <= 1e-12 sum_m |M_m z_m|
    scale = (abs(M) @ np.abs(z).ravel()).reshape(r.shape)
    back = np.abs(r - (M @ z.ravel()).reshape(r.shape))
    assert np.all(back <= 1e-12 * scale + 1e-300), np.max(back / (scale + 1e-300))
    z_ref = O.spla.spsolve(M.tocsc(), r.ravel()).reshape(r.shape)
    assert rel(z, z_ref) < 1e-8
    s.close()


@pytest.mark.parametrize("law", ["gpbld", "pb", "arr", "arrwarm", "hooke"])
def test_hardness_from_enthalpy(law):
    g, c, f = random_case(7, flow_law=law)
    G, Cc, I = O.from_case(g, c, f)
    s = make_solver(g, c, f)
    s.compute_hardav_staggered()
    np.testing.assert_allclose(s.hardness(), O.hardness_staggered(G, Cc, I), rtol=1e-12)
    s.close()


@pytest.mark.parametrize("pc,precision,ksp", [("bjacobi", "fp64", "bicgstab"), ("mg", "fp64", "bicgstab"),
                                               ("mg", "mixed", "bicgstab"), ("bjacobi", "fp64", "gmres"),
                                               ("mg", "fp64", "gmres"), ("line", "fp64", "bicgstab"),
                                               ("line", "fp64", "gmres")])
def test_linear_solve_matches_direct(pc, precision, ksp):
    """One KSPSolve at the first Picard step (zero velocity: plastic drag 1e14, the worst
    conditioning of the solve).  Both answers must have tiny true residuals and agree.
    GMRES (restart 30, classical Gram-Schmidt) runs with restarts on this system."""
    g, c, f, _ = S.build_synthetic(41, 4000e3 / 40, seed=3)
    c.ksp_rtol = 1e-14
    c.pc_type = pc
    c.precision = precision
    c.ksp_type = ksp
    G, Cc, I = O.from_case(g, c, f)
    s = make_solver(g, c, f)
    s.assemble_rhs()
    s.compute_hardav_staggered()
    vel = np.zeros((g.Mx, g.My, 2))
    s.set_initial_guess(vel)
    s.compute_nuH_staggered(c.epsilon_ssa)
    A = O.assemble_matrix(G, Cc, I, s.nuH(), s.beta())
    x_ref = O.linear_solve(A, s.rhs().ravel(), None, "direct").reshape(vel.shape)
    xd = torch.zeros((g.Mx, g.My, 2), dtype=torch.float64, device="cuda")
    its, res = s.linear_solve(xd)
    assert res <= 1e-14
    x = xd.cpu().numpy()
    b = s.rhs().ravel()
    res_gpu = np.linalg.norm(b - A @ x.ravel()) / np.linalg.norm(b)
    res_ref = np.linalg.norm(b - A @ x_ref.ravel()) / np.linalg.norm(b)
    assert res_gpu < 1e-12, (res_gpu, res_ref)
    assert rel(x, x_ref) < 1e-8, (rel(x, x_ref), res_gpu, res_ref)
    s.close()


def test_picard_iterates_match_oracle():
    """Iterate-by-iterate: nu*H -> linear solve, five Picard steps on a synthetic sheet."""
    g, c, f, _ = S.build_synthetic(33, 4000e3 / 32, seed=5)
    c.ksp_rtol = 1e-13
    G, Cc, I = O.from_case(g, c, f)
    s = make_solver(g, c, f)
    o = O.SSAFDOracle(G, Cc, I)
    o.prepare()
    s.assemble_rhs()
    s.compute_hardav_staggered()
    vel_ref = np.zeros((g.Mx, g.My, 2))
    xd = torch.zeros((g.Mx, g.My, 2), dtype=torch.float64, device="cuda")
    s.set_initial_guess(xd)
    for _ in range(5):
        s.compute_nuH_staggered(c.epsilon_ssa)
        nuH = O.compute_nuH(G, Cc, I, o.hardness, vel_ref, c.epsilon_ssa)
        np.testing.assert_allclose(s.nuH(), nuH, rtol=1e-8)
        A = O.assemble_matrix(G, Cc, I, nuH, O.beta_field(Cc, I, vel_ref))
        vel_ref = O.linear_solve(A, o.b.ravel(), None, "direct").reshape(vel_ref.shape)
        s.linear_solve(xd)
        s.set_initial_guess(xd)
        assert rel(xd.cpu().numpy(), vel_ref) < 1e-8
    s.close()


def _solve_case(g, c, f):
    s = make_solver(g, c, f)
    vel = s.solve()
    st = s.stats()
    s.close()
    return vel, st


@pytest.mark.parametrize("pc,precision,ksp", [("bjacobi", "fp64", "bicgstab"), ("mg", "fp64", "bicgstab"),
                                               ("mg", "mixed", "bicgstab"), ("mg", "fp64", "gmres"),
                                               ("line", "fp64", "bicgstab")])
@pytest.mark.parametrize("My", [61, 121])
def test_verification_i(goldens, My, pc, precision, ksp):
    g, c, f = V.build_test_i(My=My)
    c.pc_type = pc
    c.precision = precision
    c.ksp_type = ksp
    c.ssafd_relative_convergence = 5e-7
    c.ksp_rtol = 1e-12
    vel, st = _solve_case(g, c, f)
    assert st["converged"] == 1
    case = [k for k in goldens["test_i_fd"]["cases"] if k["My"] == My][0]
    r = V.report(vel, V.exact_velocity_i(g))
    for key, d in (("maxvector", 4), ("prcntavvec", 5), ("maxu", 4), ("maxv", 4), ("avu", 4), ("avv", 4)):
        assert round(r[key], d) == pytest.approx(case[key], abs=0.6 * 10 ** -d), key
    ref = O.SSAFDOracle(*O.from_case(g, c, f)).solve()
    assert rel(vel, ref) < 1e-8


@pytest.mark.parametrize("pc", ["bjacobi", "mg", "line"])
@pytest.mark.parametrize("Mx", [201, 401])
def test_verification_v_cfbc(goldens, Mx, pc):
    g, c, f = V.build_test_v(Mx)
    c.pc_type = pc
    c.ksp_rtol = 1e-13
    vel, st = _solve_case(g, c, f)
    case = [k for k in goldens["test_v_cfbc"]["cases"] if k["Mx"] == Mx][0]
    r = V.report(vel, V.exact_velocity_v(g))
    for key, d in (("maxvector", 4), ("prcntavvec", 5), ("maxu", 4), ("avu", 4)):
        assert round(r[key], d) == pytest.approx(case[key], abs=0.6 * 10 ** -d), key
    ref = O.SSAFDOracle(*O.from_case(g, c, f)).solve()
    assert rel(vel, ref) < 1e-8


@pytest.mark.parametrize("pc,ksp", [("bjacobi", "bicgstab"), ("mg", "bicgstab"), ("bjacobi", "gmres"),
                                    ("mg", "gmres"), ("line", "bicgstab")])
@pytest.mark.parametrize("M", [61, 121])
def test_verification_j(M, pc, ksp):
    """Test J with a tight KSP equals the oracle's direct solve (the golden itself
    records PETSc's rtol-1e-5 iterate; the CPU suite pins that)."""
    g, c, f = V.build_test_j(M, M)
    c.pc_type = pc
    c.ksp_type = ksp
    c.ksp_rtol = 1e-13
    vel, st = _solve_case(g, c, f)
    ref = O.SSAFDOracle(*O.from_case(g, c, f)).solve()
    assert rel(vel, ref) < 1e-8


def test_zero_diagonal_is_reported():
    """A regular cell with no coupling and no drag: the reference throws (SSAFD.cc:766-776)."""
    M = 9
    g = GridDesc(M, M, 40e3, 40e3, periodicity=0)
    c = SSAConfig(flow_law="isothermal_glen")
    f = {"thickness": np.zeros((M, M)), "surface": np.zeros((M, M)), "bed": np.full((M, M), -500.0),
         "mask": np.full((M, M), 4.0), "tauc": np.zeros((M, M))}
    c.constant_nu_strength_extension_ssa = 0.0
    c.epsilon_ssa = 0.0
    s = make_solver(g, c, f)
    with pytest.raises(ZeroDiagonal):
        s.solve()
    s.close()


@pytest.mark.parametrize("pc,precision,ksp", [("bjacobi", "fp64", "bicgstab"), ("mg", "fp64", "bicgstab"),
                                               ("mg", "mixed", "bicgstab"), ("mg", "fp64", "gmres"),
                                               ("line", "fp64", "bicgstab")])
@pytest.mark.parametrize("M", [45, 64])
def test_synthetic_solve_matches_oracle(M, pc, precision, ksp):
    """A whole SSAFD::solve of the synthetic sheet against the oracle, odd and even grid sizes
    (the multigrid aggregates wrap differently).  Pseudo-plastic till: its Picard iteration
    contracts ~25 % per step, so both solvers stop at the same iteration; with plastic till
    the nu*H change decreases ~1 % per step near 1e-4 and the stopping step is ill-posed."""
    g, c, f, _ = S.build_synthetic(M, 4000e3 / (M - 1), seed=2)
    c.do_pseudo_plastic_till = True
    c.ssafd_relative_convergence = 1e-7
    c.ksp_rtol = 1e-12
    c.pc_type = pc
    c.precision = precision
    c.ksp_type = ksp
    vel, st = _solve_case(g, c, f)
    o = O.SSAFDOracle(*O.from_case(g, c, f))
    ref = o.solve()
    assert st["converged"] == 1 and st["strategy"] == o.stats.strategy
    assert abs(st["picard_iterations"] - o.stats.picard_iterations) <= 1
    assert rel(vel, ref) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_inexact_picard_meets_the_same_tolerance(precision):
    """ksp_rtol_adaptive: early Picard iterations solve to 0.1 x the last relative nu*H
    change (at most 1e-2), the accepted iteration to ksp_rtol.  The result agrees with
    the oracle's exact-solve Picard to well inside the 1e-5 velocity bar, in the same
    number of Picard iterations, with fewer Krylov iterations than exact solves take."""
    g, c, f, _ = S.build_synthetic(45, 4000e3 / 44, seed=2)
    c.do_pseudo_plastic_till = True
    c.ssafd_relative_convergence = 1e-7
    c.ksp_rtol = 1e-10
    c.pc_type = "mg"
    c.precision = precision
    c.ksp_rtol_adaptive = True
    c.ksp_rtol_factor = 0.1
    c.ksp_rtol_max = 1e-2
    vel, st = _solve_case(g, c, f)
    o = O.SSAFDOracle(*O.from_case(g, c, f))
    ref = o.solve()
    assert st["converged"] == 1
    assert st["final_linear_residual"] <= 1e-10
    assert abs(st["picard_iterations"] - o.stats.picard_iterations) <= 1
    assert rel(vel, ref) < 1e-7
    exact_ksp = _solve_case(g, c.copy(ksp_rtol_adaptive=False), f)[1]["ksp_iterations"]
    assert st["ksp_iterations"] < 0.8 * exact_ksp


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_launch_modes_agree_bitwise(precision):
    """graphs = 2 (graph-resident loops), 1 (replayed iteration graphs) and 0 (direct
    launches) run the same kernels in the same order: identical velocities and counts."""
    g, c, f, _ = S.build_synthetic(41, 4000e3 / 40, seed=8)
    c.pc_type = "mg"
    c.precision = precision
    c.ksp_rtol = 1e-8
    c.ksp_rtol_adaptive = True
    c.ksp_rtol_factor = 1.0
    c.ksp_rtol_max = 1e-1
    out = {}
    for mode in (2, 1, 0):
        vel, st = _solve_case(g, c.copy(graphs=mode), f)
        out[mode] = (vel, st["picard_iterations"], st["ksp_iterations"], st["refinement_steps"])
    for mode in (1, 0):
        np.testing.assert_array_equal(out[mode][0], out[2][0])
        assert out[mode][1:] == out[2][1:]


def test_ksp_failure_falls_back_and_is_reported():
    """A Krylov budget too small to converge (FP64 path): the failure switches
    preconditioner (multigrid -> block Jacobi, as the reference switches to ASM,
    SSAFD.cc:929-958), the retry fails too and SSAFD::solve reports KSPFailure; the handle
    stays usable and a solve with a normal budget afterwards succeeds.  (With precision
    mixed, ksp_max_it bounds each inner FP32 solve and the FP64 refinement goes on.)"""
    from pism_b200.ssa import KSPFailure
    g, c, f, _ = S.build_synthetic(41, 4000e3 / 40, seed=9)
    c.pc_type = "mg"
    c.precision = "fp64"
    c.ksp_rtol = 1e-10
    c.ksp_max_it = 2
    s = make_solver(g, c, f)
    with pytest.raises(KSPFailure):
        s.solve()
    s.set_config(c.copy(ksp_max_it=10000))
    s.set_initial_guess(np.zeros((g.Mx, g.My, 2)))
    vel = s.solve()
    st = s.stats()
    assert st["converged"] == 1 and np.all(np.isfinite(vel))
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lagged_coarse_levels_meet_the_same_tolerance(precision):
    """mg_rebuild_rtol: the multigrid coarse levels are rebuilt only once the summed relative
    nu*H change reaches 0.05; the answer agrees with the oracle's exact-solve Picard as the
    non-lagged solve does, in the same number of Picard iterations, with fewer coarse
    builds than Picard iterations."""
    g, c, f, _ = S.build_synthetic(45, 4000e3 / 44, seed=2)
    c.do_pseudo_plastic_till = True
    c.ssafd_relative_convergence = 1e-7
    c.ksp_rtol = 1e-10
    c.pc_type = "mg"
    c.precision = precision
    c.mg_rebuild_rtol = 0.05
    vel, st = _solve_case(g, c, f)
    o = O.SSAFDOracle(*O.from_case(g, c, f))
    ref = o.solve()
    assert st["converged"] == 1 and st["final_linear_residual"] <= 1e-10
    assert abs(st["picard_iterations"] - o.stats.picard_iterations) <= 1
    assert 1 <= st["mg_rebuilds"] < st["picard_iterations"]
    assert rel(vel, ref) < 1e-7


@pytest.mark.parametrize("shape,precision", [((201, 201), "mixed"), ((64, 64), "fp64"), ((45, 44), "mixed"),
                                              ("test_i", "fp64")])
def test_small_level_cycles_agree_bitwise(shape, precision):
    """The multigrid's small levels staged from L2 at every step (mg_small_kernel 0) and held
    by every CTA as a block of every level in shared memory (1): the same arithmetic per cell
    in the same order, so the same velocities and counts, bit for bit."""
    if shape == "test_i":
        g, c, f = V.build_test_i(My=201)
        c.ssafd_relative_convergence = 5e-7
        c.ksp_rtol = 1e-12
    else:
        g, c, f, _ = S.build_synthetic(shape[0], 4000e3 / (shape[0] - 1), seed=6)
        c.ksp_rtol = 1e-8
    c = c.copy(pc_type="mg", precision=precision)
    out = {}
    for k in (0, 1):
        vel, st = _solve_case(g, c.copy(mg_small_kernel=k), f)
        out[k] = (vel, st["picard_iterations"], st["ksp_iterations"], st["refinement_steps"])
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1:] == out[1][1:]


@pytest.mark.parametrize("shape,precision", [((201, 201), "mixed"), ((401, 401), "mixed"), ((201, 201), "fp64")])
def test_wide_cluster_cycle_meets_the_same_tolerances(shape, precision):
    """mg_small_kernel 2 (the cluster also cycles the level of <= 16384 cells) against 0: the
    same preconditioner up to the order of one sum, so the same Picard count, Krylov counts
    within a few, and answers that agree far inside the solve's tolerance"""
    g, c, f, _ = S.build_synthetic(shape[0], 4000e3 / (shape[0] - 1), seed=6)
    c = c.copy(pc_type="mg", precision=precision, ksp_rtol=1e-8)
    out = {}
    for k in (0, 2):
        vel, st = _solve_case(g, c.copy(mg_small_kernel=k), f)
        assert st["converged"] == 1
        out[k] = (vel, st)
    assert out[0][1]["picard_iterations"] == out[2][1]["picard_iterations"]
    assert abs(out[0][1]["ksp_iterations"] - out[2][1]["ksp_iterations"]) <= 0.05 * out[0][1]["ksp_iterations"] + 3
    assert rel(out[2][0], out[0][0]) < 1e-6


@pytest.mark.parametrize("shape,graphs", [((201, 201), 3), ((161, 131), 2), ((130, 97), 0), ((45, 44), 3),
                                           ("test_i", 3)])
def test_apply_kernels_agree_bitwise(shape, graphs):
    """Each FP32 V-cycle's fine-level pass fused with the operator apply that follows it
    (mixed_apply_kernel 2: the halo of the smoothed iterate recomputed per tile) against the
    apply kernel of its own with plain (0) and bulk-copy staged (1) tile loads: the same
    arithmetic per cell and the same sums in the same order, so the same velocities and counts,
    bit for bit -- on ragged tiles, periodic wrap at the grid's edges and Dirichlet rows."""
    if shape == "test_i":
        g, c, f = V.build_test_i(My=201)
        c.ssafd_relative_convergence = 5e-7
        c.ksp_rtol = 1e-12
    else:
        Mx, My = shape
        g, c, f, _ = S.build_synthetic(Mx, 4000e3 / (Mx - 1), seed=6)
        if My != Mx:
            g = GridDesc(Mx, My, g.Lx, g.Lx * (My - 1) / (Mx - 1), periodicity=0, z=g.z)
            f = {k: (v[:Mx, :My] if isinstance(v, np.ndarray) else v) for k, v in f.items()}
        c.ksp_rtol = 1e-8
        c.do_pseudo_plastic_till = True
    c = c.copy(pc_type="mg", precision="mixed", graphs=graphs)
    out = {}
    for k in (0, 1, 2):
        vel, st = _solve_case(g, c.copy(mixed_apply_kernel=k), f)
        out[k] = (vel, st["picard_iterations"], st["ksp_iterations"], st["refinement_steps"])
    for k in (1, 2):
        np.testing.assert_array_equal(out[0][0], out[k][0])
        assert out[0][1:] == out[k][1:]


@pytest.mark.parametrize("shape", [(161, 131), (130, 97)])
def test_mixed_solve_on_grids_with_staged_tiles(shape):
    """Grids wide enough for the FP32 apply kernels to stage interior tiles by bulk copies
    (tile columns 32 .. My - 36) next to the plain-loaded edge columns: the mixed-precision
    linear solve against a direct solve, and a whole solve against the oracle."""
    Mx, My = shape
    g, c, f, _ = S.build_synthetic(Mx, 4000e3 / (Mx - 1), seed=12)
    g = GridDesc(Mx, My, g.Lx, g.Lx * (My - 1) / (Mx - 1), periodicity=0, z=g.z)
    f = {k: (v[:Mx, :My] if isinstance(v, np.ndarray) else v) for k, v in f.items()}
    c = c.copy(pc_type="mg", precision="mixed", ksp_rtol=1e-12, do_pseudo_plastic_till=True,
               ssafd_relative_convergence=1e-7)
    G, Cc, I = O.from_case(g, c, f)
    s = make_solver(g, c, f)
    s.assemble_rhs()
    s.compute_hardav_staggered()
    s.set_initial_guess(np.zeros((Mx, My, 2)))
    s.compute_nuH_staggered(c.epsilon_ssa)
    A = O.assemble_matrix(G, Cc, I, s.nuH(), s.beta())
    x_ref = O.linear_solve(A, s.rhs().ravel(), None, "direct").reshape((Mx, My, 2))
    xd = torch.zeros((Mx, My, 2), dtype=torch.float64, device="cuda")
    its, res = s.linear_solve(xd)
    assert res <= 1e-12
    x = xd.cpu().numpy()
    b = s.rhs().ravel()
    res_gpu = np.linalg.norm(b - A @ x.ravel()) / np.linalg.norm(b)
    # the first Picard step's system (plastic drag at zero velocity) has a condition number
    # near 1e5 on these grids: the true residual is the sharp check, the error follows it
    assert res_gpu < 1e-11, res_gpu
    assert rel(x, x_ref) < 1e-6, (rel(x, x_ref), res_gpu)
    s.close()
    vel, st = _solve_case(g, c, f)
    o = O.SSAFDOracle(G, Cc, I)
    ref = o.solve()
    assert st["converged"] == 1 and abs(st["picard_iterations"] - o.stats.picard_iterations) <= 1
    assert rel(vel, ref) < 1e-7
