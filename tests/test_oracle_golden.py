"""The CPU oracle against the reference's own golden outputs (CPU only).

Pins: exactTestsIJ.c values (computed by the reference's C file), the flow-law
tables of test/regression/test_2x.sh, and the verification error tables of
test/regression/ssa/*.sh and doc/verif/I_userman_may2012.nc.
"""
import numpy as np
import pytest

from pism_b200 import verification as V
from oracle import ssafd_oracle as O

KEYS = ["maxvector", "prcntavvec", "maxu", "maxv", "avu", "avv"]
DIGITS = {"maxvector": 4, "prcntavvec": 5, "maxu": 4, "maxv": 4, "avu": 4, "avv": 4}  # %11.4f%13.5f%10.4f...


def assert_table(report, golden):
    for k in KEYS:
        assert round(report[k], DIGITS[k]) == pytest.approx(golden[k], abs=0.6 * 10 ** -DIGITS[k]), k


def test_exact_i_matches_reference_c(goldens):
    pts = np.array(goldens["exact_i"]["points"])
    bed, tauc, u, v = V.exact_i(goldens["exact_i"]["m"], pts[:, 0], pts[:, 1])
    np.testing.assert_allclose(np.stack([bed, tauc, u, v], 1), pts[:, 2:], rtol=1e-13, atol=1e-300)


def test_exact_j_matches_reference_c(goldens):
    pts = np.array(goldens["exact_j"]["points"])
    H, nu, u, v = V.exact_j(pts[:, 0], pts[:, 1])
    np.testing.assert_allclose(np.stack([H, nu, u, v], 1), pts[:, 2:], rtol=1e-12, atol=1e-22)


@pytest.mark.parametrize("law", ["gpbld", "pb", "hooke", "arr"])
def test_flow_law_tables(goldens, law):
    """flowlaw_test.cc: flow = A(E, p) * sigma^(n-1) at p = pressure(2000 m)."""
    t = goldens["flow_tables"][law]
    cfg = O.Config(flow_law=law)
    p = float(O.ec_pressure(cfg, 2000.0))
    assert p == pytest.approx(t["pressure"], rel=1e-3)
    for sigma, T, omega, flow in t["rows"]:
        E = O.ec_enthalpy(cfg, T, omega, p)
        if law == "arr":   # PatersonBuddCold::flow_from_temp uses the absolute temperature
            A = cfg.Paterson_Budd_A_cold * np.exp(-cfg.Paterson_Budd_Q_cold / (cfg.ideal_gas_constant * T))
        else:
            A = O.softness(cfg, E, p)
        assert float(A * sigma ** 2) == pytest.approx(flow, rel=6e-7)


@pytest.mark.parametrize("k", [0, 1])
def test_verification_i(goldens, k):
    case = goldens["test_i_fd"]["cases"][k]
    g, c, f = V.build_test_i(My=case["My"])
    c.ssafd_relative_convergence = goldens["test_i_fd"]["options"]["ssa_rtol"]
    o = O.SSAFDOracle(*O.from_case(g, c, f))
    vel = o.solve()
    assert o.stats.converged and o.stats.strategy == 0
    assert_table(V.report(vel, V.exact_velocity_i(g)), case)


@pytest.mark.parametrize("k", [0, 1])
def test_verification_j_petsc_like(goldens, k):
    """Test J converges in one Picard step, so the golden records PETSc's inexact KSP:
    reproduced by the oracle's GMRES(30) + block-Jacobi ILU(0) over the 2-rank DMDA split."""
    case = goldens["test_j_fd"]["cases"][k]
    g, c, f = V.build_test_j(case["Mx"], case["My"])
    o = O.SSAFDOracle(*O.from_case(g, c, f), linear="petsc", ksp_rtol=1e-5, nranks=2)
    vel = o.solve()
    assert o.stats.picard_iterations == 1
    assert_table(V.report(vel, V.exact_velocity_j(g)), case)


@pytest.mark.parametrize("k", [0, 1])
def test_verification_v_cfbc(goldens, k):
    case = goldens["test_v_cfbc"]["cases"][k]
    g, c, f = V.build_test_v(case["Mx"], case["My"])
    o = O.SSAFDOracle(*O.from_case(g, c, f))
    vel = o.solve()
    assert o.stats.converged
    assert_table(V.report(vel, V.exact_velocity_v(g)), case)


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_verification_i_user_manual(goldens, k):
    t = goldens["test_i_userman"]
    My = int(round(240e3 / t["dy"][k])) + 1
    g, c, f = V.build_test_i(My=My)
    c.ssafd_relative_convergence = t["options"]["ssa_rtol"]
    vel = O.SSAFDOracle(*O.from_case(g, c, f)).solve()
    r = V.report(vel, V.exact_velocity_i(g))
    assert r["maxvector"] == pytest.approx(t["max_velocity"][k], rel=2e-4)
    assert r["prcntavvec"] == pytest.approx(t["relative_velocity"][k], rel=2e-4)
    assert r["avu"] == pytest.approx(t["average_u"][k], rel=2e-4)
    assert r["maxv"] == pytest.approx(t["maximum_v"][k], rel=1e-3)


def test_petsc_like_matches_direct_on_tight_tolerance():
    """The PETSc-like KSP and the direct solve agree when the KSP is tight."""
    g, c, f = V.build_test_i(My=61)
    G, Cc, I = O.from_case(g, c, f)
    o = O.SSAFDOracle(G, Cc, I)
    o.prepare()
    vel = np.zeros((G.Mx, G.My, 2))
    nuH = O.compute_nuH(G, Cc, I, o.hardness, vel, Cc.epsilon_ssa)
    A = O.assemble_matrix(G, Cc, I, nuH, O.beta_field(Cc, I, vel))
    x_direct = O.linear_solve(A, o.b.ravel(), vel.ravel(), "direct")
    x_petsc, its, reason = O.petsc_gmres_bjacobi(A, o.b.ravel(), vel.ravel(), G.Mx, G.My, nranks=2,
                                                 rtol=1e-13)
    assert reason == 0
    np.testing.assert_allclose(x_petsc, x_direct, rtol=1e-7, atol=1e-9 * np.abs(x_direct).max())


def test_apply_stencil_equals_assembled_matrix():
    """The stencil-wise apply and the assembled CSR matrix are the same operator."""
    rng = np.random.default_rng(0)
    g, c, f = V.build_test_v(41, 5)
    G, Cc, I = O.from_case(g, c, f)
    nuH = rng.uniform(1e14, 1e17, (G.Mx, G.My, 2))
    beta = rng.uniform(0, 1e10, (G.Mx, G.My))
    A = O.assemble_matrix(G, Cc, I, nuH, beta)
    x = rng.standard_normal((G.Mx, G.My, 2))
    y = O.apply_stencil(G, Cc, I, nuH, beta, x)
    np.testing.assert_allclose(y.ravel(), A @ x.ravel(), rtol=1e-12, atol=1e-9 * np.abs(y).max())


def test_line_block_recurrences_equal_the_direct_solve():
    """The line preconditioner's block LU recurrences (the device algorithm) solve exactly
    the line-tridiagonal part of A, periodic wrap across the line ends dropped."""
    rng = np.random.default_rng(1)
    g, c, f = V.build_test_v(13, 7)
    G, Cc, I = O.from_case(g, c, f)
    nuH = rng.uniform(1e14, 1e17, (G.Mx, G.My, 2))
    beta = rng.uniform(0, 1e10, (G.Mx, G.My))
    A = O.assemble_matrix(G, Cc, I, nuH, beta)
    M = O.line_block_part(G, A)
    assert M.nnz < A.nnz
    r = rng.standard_normal((G.Mx, G.My, 2))
    z = O.line_block_solve(G, A, r)
    np.testing.assert_allclose((M @ z.ravel()).reshape(r.shape), r, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(O.line_block_lu_solve(G, A, r), z, rtol=1e-9, atol=1e-12 * np.abs(z).max())
    # no coupling between lines: a right-hand side on one line stays on it
    r1 = np.zeros_like(r)
    r1[3] = r[3]
    z1 = O.line_block_solve(G, A, r1)
    assert np.all(z1[:3] == 0) and np.all(z1[4:] == 0)
