"""GPU parity on the configurations the targets are stated on, through the C-ABI.

* The 801 x 801 benchmark sheet (plastic till, FP64): Picard iterates one by one against
  the oracle, the full-size stencil against the oracle's assembled matrix.
* Plastic-till whole solves at 201^2 and 401^2 that stop at a fixed Picard count (a
  tolerance placed between the oracle's own iterations K - 1 and K, with a margin).
* Verification test I on its configuration grid (Mx = 5, My = 201) at the reference's
  default tolerances and at the user manual's tight ones.
* The strategy ladder of SSAFD::solve (SSAFD.cc:869-924, 1122-1155): under-relaxation and
  over-regularisation, each converging, and the silent end when all strategies fail.
* Fracture-induced softening (SSAFD.cc:1282-1310), the basal frictional heating
  (ShallowStressBalance.cc:179-205) and the solver's fused nu*H norms (SSAFD.cc:1170-1189).

Tolerances: stage values 1e-12 relative (as in test_gpu_parity.py); velocities 1e-8
relative L2 with tight KSP tolerances on both sides.
"""
import os

import numpy as np
import pytest

from pism_b200 import verification as V, synthetic as S
from oracle import ssafd_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200.ssa import SSAFD  # noqa: E402

from test_gpu_parity import make_solver, random_case, rel  # noqa: E402

NTHREADS = min(16, os.cpu_count() or 1)


def _sheet_801():
    """the 801 x 801 benchmark sheet (seed 0, 5 km, plastic till) of bench.py"""
    g, c, f, _ = S.build_synthetic(801, 4000e3 / 800, seed=0)
    return g, c, f


def test_config2_801_picard_iterates_match_oracle():
    """Three Picard iterations on the 801^2 benchmark sheet, iterate by iterate: nu*H at the
    GPU's own velocity against the oracle's at the oracle's velocity, the GPU's linear solve
    (FP64 BiCGStab + multigrid to 1e-13) against the oracle's PETSc-like GMRES(30) + block
    Jacobi ILU(0) to 1e-13, each from the previous iterate.  At the first step the GPU's
    matrix-free operator is also checked row by row against the oracle's assembled matrix."""
    g, c, f = _sheet_801()
    c.pc_type = "mg"
    c.ksp_rtol = 1e-13
    G, Cc, I = O.from_case(g, c, f)
    s = make_solver(g, c, f)
    o = O.SSAFDOracle(G, Cc, I)
    o.prepare()
    s.assemble_rhs()
    s.compute_hardav_staggered()
    np.testing.assert_allclose(s.rhs(), o.b, rtol=1e-12, atol=1e-9 * np.abs(o.b).max())
    reg = c.epsilon_ssa
    M = g.Mx
    vel_ref = np.zeros((M, M, 2))
    xd = torch.zeros((M, M, 2), dtype=torch.float64, device="cuda")
    s.set_initial_guess(xd)
    b = o.b.ravel()
    for k in range(3):
        s.compute_nuH_staggered(reg)
        nuH_ref = O.compute_nuH(G, Cc, I, o.hardness, vel_ref, reg)
        beta_ref = O.beta_field(Cc, I, vel_ref)
        assert rel(s.nuH(), nuH_ref) < (1e-12 if k == 0 else 1e-8), k
        assert rel(s.beta(), beta_ref) < (1e-12 if k == 0 else 1e-8), k
        A = O.assemble_matrix(G, Cc, I, nuH_ref, beta_ref)
        if k == 0:
            rng = np.random.default_rng(3)
            x = rng.normal(0, 1e-5, (M, M, 2))
            yd = torch.empty_like(xd)
            s.apply(torch.tensor(x, device="cuda"), yd)
            torch.cuda.synchronize()
            scale = (abs(A) @ np.abs(x).ravel()).reshape(x.shape)
            back = np.abs(yd.cpu().numpy() - (A @ x.ravel()).reshape(x.shape))
            assert np.all(back <= 1e-12 * scale + 1e-300), np.max(back / (scale + 1e-300))
        x_ref, its_ref, reason = O.petsc_gmres_bjacobi(A, b, vel_ref.ravel(), M, M, nranks=NTHREADS, rtol=1e-13,
                                                       nthreads=NTHREADS)
        assert reason == 0
        vel_ref = x_ref.reshape(vel_ref.shape)
        its, res = s.linear_solve(xd)
        assert res <= 1e-13
        s.set_initial_guess(xd)
        x_gpu = xd.cpu().numpy()
        # the GPU iterate's backward error in the oracle's matrix, then the forward agreement
        assert np.linalg.norm(b - A @ x_gpu.ravel()) / np.linalg.norm(b) < 1e-12, k
        assert rel(x_gpu, vel_ref) < 1e-8, (k, rel(x_gpu, vel_ref))
    s.close()


def _fixed_count_tolerance(history, K):
    """a Picard tolerance at which the oracle's iteration stops exactly at K: between the
    relative change of iteration K and the smallest one before it, with >= 2 % margin"""
    ratios = [ch / nm for nm, ch in history]
    last, before = ratios[K - 1], min(ratios[:K - 1])
    assert last * 1.02 < before / 1.02, (last, before)
    return float(np.sqrt(last * before))


@pytest.mark.parametrize("M,K", [(201, 12), (401, 12)])
def test_plastic_till_whole_solve_fixed_picard_count(M, K):
    """pism_gpu_ssa_solve (graph-resident loops, FP64 BiCGStab + multigrid to 1e-13) on a
    plastic-till synthetic sheet against K Picard iterations of the oracle (its PETSc-like
    KSP to 1e-13).  The GPU's Picard tolerance is placed between the oracle's relative nu*H
    changes of iterations K - 1 and K, so the GPU solve must stop exactly at K."""
    g, c, f, _ = S.build_synthetic(M, 4000e3 / (M - 1), seed=4)
    c.pc_type = "mg"
    c.ksp_rtol = 1e-13
    G, Cc, I = O.from_case(g, c, f)
    o = O.SSAFDOracle(G, Cc.copy(max_iterations_ssafd=K, ssafd_relative_convergence=1e-30), I, linear="petsc",
                      ksp_rtol=1e-13, nranks=NTHREADS, nthreads=NTHREADS)
    o.prepare()
    with pytest.raises(O.PicardFailure):
        o.picard_manager(Cc.epsilon_ssa, 1.0)
    ref = o.velocity
    c.ssafd_relative_convergence = _fixed_count_tolerance(o.stats.history, K)
    s = make_solver(g, c, f)
    vel = s.solve()
    st = s.stats()
    s.close()
    assert st["converged"] == 1 and st["strategy"] == 0 and st["picard_iterations"] == K
    assert rel(vel, ref) < 1e-8, rel(vel, ref)
    # the last Picard test's norms: |nu*H| to 1e-10, the change (a difference of iterates) to 1e-6
    norm, change = o.stats.history[K - 1]
    assert st["nuH_norm"] == pytest.approx(norm, rel=1e-10)
    assert st["nuH_norm_change"] == pytest.approx(change, rel=1e-6)


def test_config1_test_i_reference_default_tolerances(goldens):
    """Configuration 1 as stated: test I on Mx = 5, My = 201 with the reference's default
    Picard and KSP tolerances (ssa_rtol 1e-4, KSP rtol 1e-5), the plain FP64 set-up
    (BiCGStab + block Jacobi).  Both the GPU and the oracle stop the Picard iteration at the
    same default test; the GPU's inexact linear solves (relative residual 1e-5 per Picard
    iteration) against the oracle's direct solves leave the answers 1e-6 apart at most
    (7.6e-8 measured on a B200; the oracle's own PETSc-like GMRES at 1e-5 is 3.5e-3 from its
    direct solve).  The error table against the exact solution is reported."""
    g, c, f = V.build_test_i(My=201)
    assert c.ssafd_relative_convergence == 1e-4 and c.ksp_rtol == 1e-5
    s = make_solver(g, c, f)
    vel = s.solve()
    st = s.stats()
    s.close()
    o = O.SSAFDOracle(*O.from_case(g, c, f))
    ref = o.solve()
    assert st["converged"] == 1 and st["strategy"] == 0
    assert abs(st["picard_iterations"] - o.stats.picard_iterations) <= 3
    assert rel(vel, ref) < 1e-6, rel(vel, ref)
    r = V.report(vel, V.exact_velocity_i(g))
    r_ref = V.report(ref, V.exact_velocity_i(g))
    print(f"test I 5x201 defaults: GPU picard {st['picard_iterations']} maxvector {r['maxvector']:.4f} "
          f"(oracle {o.stats.picard_iterations}, {r_ref['maxvector']:.4f}), rel L2 vs oracle {rel(vel, ref):.2e}")


@pytest.mark.parametrize("pc,ksp", [("bjacobi", "bicgstab"), ("mg", "gmres")])
def test_config1_test_i_user_manual_record(goldens, pc, ksp):
    """Test I on Mx = 5, My = 201 at the tolerances of the user manual's verification runs
    (ssa_rtol 5e-7, KSP 1e-12): the error table of doc/verif/I_userman_may2012.nc at
    dy = 1200 m (to 2e-4 relative, as the CPU suite pins the oracle) and the oracle's
    velocities to 1e-8."""
    t = goldens["test_i_userman"]
    k = t["dy"].index(1200.0)
    g, c, f = V.build_test_i(My=201)
    c.ssafd_relative_convergence = t["options"]["ssa_rtol"]
    c.ksp_rtol = t["options"]["ksp_rtol"]
    c.pc_type = pc
    c.ksp_type = ksp
    s = make_solver(g, c, f)
    vel = s.solve()
    st = s.stats()
    s.close()
    assert st["converged"] == 1
    r = V.report(vel, V.exact_velocity_i(g))
    assert r["maxvector"] == pytest.approx(t["max_velocity"][k], rel=2e-4)
    assert r["prcntavvec"] == pytest.approx(t["relative_velocity"][k], rel=2e-4)
    assert r["avu"] == pytest.approx(t["average_u"][k], rel=2e-4)
    assert r["maxv"] == pytest.approx(t["maximum_v"][k], rel=1e-3)
    ref = O.SSAFDOracle(*O.from_case(g, c, f)).solve()
    assert rel(vel, ref) < 1e-8


# (pseudo-plastic, epsilon_ssa, max_iterations_ssafd, Picard tolerance) -> the oracle's ladder
LADDER = {
    # strategy 0 fails within 12 iterations; the under-relaxed strategy 1 converges at 12
    # (relative change 8.9e-4 < 1e-3 after 1.19e-3)
    "underrelaxation": (True, 1e15, 12, 1e-3),
    # strategies 0 and 1 fail within 2 iterations; an over-regularised attempt converges
    # (relative change 3.4e-4 against >= 2.3e-3 before)
    "regularization": (False, 1e19, 2, 1e-3),
    # every strategy fails: the reference's loop ends silently (SSAFD.cc:882-911)
    "all_fail": (True, 1e13, 4, 1e-3),
}


@pytest.mark.parametrize("name", sorted(LADDER))
def test_strategy_ladder_matches_oracle(name):
    """Picard failures forced by a small max_iterations_ssafd: the GPU runs the reference's
    strategies (under-relaxation SSAFD.cc:889-897 with SSAFD.cc:1061-1064, then nu*H
    over-regularisation x 4 up to five times, SSAFD.cc:1122-1155) and ends where the oracle
    ends: same strategy, same convergence flag, same Picard count of the last attempt and
    velocities to 1e-8 (KSP 1e-13 on the GPU, direct solves in the oracle)."""
    pseudo, reg, K, rtol = LADDER[name]
    g, c, f, _ = S.build_synthetic(33, 4000e3 / 32, seed=5)
    c = c.copy(do_pseudo_plastic_till=pseudo, epsilon_ssa=reg, max_iterations_ssafd=K,
               ssafd_relative_convergence=rtol, ksp_rtol=1e-13, pc_type="mg")
    o = O.SSAFDOracle(*O.from_case(g, c, f))
    ref = o.solve()
    s = make_solver(g, c, f)
    vel = s.solve()
    st = s.stats()
    s.close()
    expect = {"underrelaxation": (1, True), "regularization": (2, True), "all_fail": (2, False)}[name]
    assert (o.stats.strategy, bool(o.stats.converged)) == expect
    assert st["strategy"] == o.stats.strategy
    assert bool(st["converged"]) == bool(o.stats.converged)
    assert st["picard_iterations"] == o.stats.picard_iterations
    assert rel(vel, ref) < 1e-8, rel(vel, ref)


@pytest.mark.parametrize("cfbc", [False, True])
def test_fracture_softening_matches_oracle(cfbc):
    """SSAFD::fracture_induced_softening (SSAFD.cc:1282-1310): the staggered hardness scaled
    by (1 - (1 - epsilon) phi)^(-n) ^ (-1/n) with phi the face average of the fracture
    density, for isothermal and enthalpy-dependent flow laws."""
    for law in ("isothermal_glen", "gpbld"):
        g, c, f = random_case(41 + cfbc, cfbc=cfbc, flow_law=law)
        c.do_fracture_density = True
        c.fracture_density_softening_lower_limit = 0.3
        f["fracture_density"] = np.random.default_rng(9).uniform(0.0, 1.0, (g.Mx, g.My))
        G, Cc, I = O.from_case(g, c, f)
        s = make_solver(g, c, f)
        s.compute_hardav_staggered()
        hard = O.hardness_staggered(G, Cc, I)
        unsoftened = O.hardness_staggered(G, Cc.copy(do_fracture_density=False), I)
        assert np.any(np.abs(hard - unsoftened) > 1e-3 * np.abs(unsoftened))   # softening acts
        np.testing.assert_allclose(s.hardness(), hard, rtol=1e-12)
        s.close()


@pytest.mark.parametrize("name", ["plain", "cfbc", "pseudo_subgl"])
def test_fused_norms_and_frictional_heating_match_oracle(name):
    """One Picard iteration from a random initial velocity (a tolerance that every first
    test meets): the solver's fused nu*H norms (SSAFD::compute_nuH_norm, SSAFD.cc:1170-1189,
    over the ghosted arrays) against the oracle's nuH_norm of the GPU's nu*H before and
    after, and compute_basal_frictional_heating (ShallowStressBalance.cc:179-205) against
    the oracle's at the GPU's velocity."""
    if name == "cfbc":
        # verification test V (a calving front with the CFBC stencil); random -cfbc mask
        # patterns nearly always leave an isolated icy cell with a zero diagonal, which the
        # solve reports as the reference does (SSAFD.cc:766-776; the oracle finds the same cell)
        g, c, f = V.build_test_v(201)
    else:
        kw = {"plain": dict(), "pseudo_subgl": dict(pseudo=True, sub_gl=True)}[name]
        g, c, f = random_case(31 + len(name), bc=False, **kw)
    vel0 = np.random.default_rng(8).normal(0, 3e-6, (g.Mx, g.My, 2))
    c.max_iterations_ssafd = 1
    c.ssafd_relative_convergence = 1e30
    c.ksp_rtol = 1e-10
    G, Cc, I = O.from_case(g, c, f)
    s = make_solver(g, c, f)
    s.compute_hardav_staggered()
    nuH0 = O.compute_nuH(G, Cc, I, O.hardness_staggered(G, Cc, I), vel0, c.epsilon_ssa)
    s.set_initial_guess(vel0)
    vel = s.solve()
    st = s.stats()
    assert st["picard_iterations"] == 1 and st["converged"] == 1
    nuH1 = s.nuH()
    np.testing.assert_allclose(nuH1, O.compute_nuH(G, Cc, I, O.hardness_staggered(G, Cc, I), vel, c.epsilon_ssa),
                               rtol=1e-12)
    norm, change = O.nuH_norm(G, nuH1, nuH0)
    assert st["nuH_norm"] == pytest.approx(norm, rel=1e-12)
    assert st["nuH_norm_change"] == pytest.approx(change, rel=1e-10)
    heat = O.basal_frictional_heating(Cc, I, vel)
    np.testing.assert_allclose(s.basal_frictional_heating(), heat, rtol=1e-12, atol=1e-12 * np.abs(heat).max())
    assert name == "cfbc" or np.abs(heat).max() > 0   # test V's shelf is all afloat: no friction
    s.close()
