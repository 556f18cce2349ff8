"""The timed CPU baseline on CPU: the native restatement of SSAFD's Picard loop
(oracle/ssafd_cpu.cc) against the Python oracle's, and the bench's whole-solve estimate
from a sample of Picard iterations."""
import importlib.util
import os

import numpy as np
import pytest

from pism_b200 import synthetic as S, verification as V
from oracle import ssafd_oracle as O

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_cpu", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _python_picard(G, Cc, I, K, nranks, vel0=None):
    o = O.SSAFDOracle(G, Cc.copy(max_iterations_ssafd=K, ssafd_relative_convergence=1e-30), I, linear="petsc",
                      ksp_rtol=1e-8, nranks=nranks, nthreads=nranks)
    o.prepare()
    if vel0 is not None:
        o.set_initial_guess(vel0)
    with pytest.raises(O.PicardFailure):
        o.picard_manager(Cc.epsilon_ssa, 1.0)
    return o


@pytest.mark.parametrize("pseudo", [False, True])
def test_native_picard_equals_python_oracle(pseudo):
    """four Picard iterations of the synthetic sheet: the native loop (C++ nu*H, drag and
    assembly in PETSc's order, the same GMRES) and the Python oracle give the same iterates
    and norms to rounding"""
    g, c, f, _ = S.build_synthetic(33, 4000e3 / 32, seed=5)
    c.do_pseudo_plastic_till = pseudo
    G, Cc, I = O.from_case(g, c, f)
    o = _python_picard(G, Cc, I, 4, nranks=4)
    vel, info = O.picard_native(G, Cc, I, o.hardness, o.b, np.zeros((33, 33, 2)), Cc.epsilon_ssa, nranks=4,
                                nthreads=4, ksp_rtol=1e-8, max_iterations=4, picard_rtol=1e-30)
    assert info["status"] == 1 and info["picard_iterations"] == 4
    assert np.linalg.norm(vel - o.velocity) <= 1e-12 * np.linalg.norm(o.velocity)
    norm, change = o.stats.history[-1]
    assert info["nuH_norm"] == pytest.approx(norm, rel=1e-12)
    assert info["nuH_norm_change"] == pytest.approx(change, rel=1e-9)
    assert len(info["ksp_iterations"]) == 4 and min(info["ksp_iterations"]) > 0


def test_native_picard_with_dirichlet_rows_and_underrelaxation():
    """verification test I (Dirichlet rows on every edge, scaled identity rows) with the
    under-relaxation of strategy 1, against the Python oracle"""
    g, c, f = V.build_test_i(My=61)
    G, Cc, I = O.from_case(g, c, f)
    o = O.SSAFDOracle(G, Cc.copy(max_iterations_ssafd=3, ssafd_relative_convergence=1e-30), I, linear="petsc",
                      ksp_rtol=1e-8, nranks=2, nthreads=2)
    o.prepare()
    with pytest.raises(O.PicardFailure):
        o.picard_manager(Cc.epsilon_ssa, 0.8)
    vel, info = O.picard_native(G, Cc, I, o.hardness, o.b, np.zeros((G.Mx, G.My, 2)), Cc.epsilon_ssa,
                                underrelax=0.8, nranks=2, nthreads=2, ksp_rtol=1e-8, max_iterations=3,
                                picard_rtol=1e-30)
    assert np.linalg.norm(vel - o.velocity) <= 1e-12 * np.linalg.norm(o.velocity)
    assert info["nuH_norm"] == pytest.approx(o.stats.history[-1][0], rel=1e-12)


def test_native_picard_stops_at_the_picard_test():
    """with a reachable tolerance the native loop stops where the Python oracle's does"""
    g, c, f, _ = S.build_synthetic(33, 4000e3 / 32, seed=5)
    c.do_pseudo_plastic_till = True
    c.ssafd_relative_convergence = 1e-3
    G, Cc, I = O.from_case(g, c, f)
    o = O.SSAFDOracle(G, Cc, I, linear="petsc", ksp_rtol=1e-8, nranks=2, nthreads=2)
    o.prepare()
    o.picard_manager(Cc.epsilon_ssa, 1.0)
    vel, info = O.picard_native(G, Cc, I, o.hardness, o.b, np.zeros((33, 33, 2)), Cc.epsilon_ssa, nranks=2,
                                nthreads=2, ksp_rtol=1e-8)
    assert info["status"] == 0 and info["picard_iterations"] == o.stats.picard_iterations


def test_native_picard_refuses_what_it_does_not_restate():
    g, c, f, _ = S.build_synthetic(17, 4000e3 / 16, seed=1)
    c.calving_front_stress_boundary_condition = True
    G, Cc, I = O.from_case(g, c, f)
    with pytest.raises(ValueError):
        O.picard_native(G, Cc, I, np.ones((17, 17, 2)), np.zeros((17, 17, 2)), np.zeros((17, 17, 2)), 1e13)


def test_whole_solve_estimate_scales_the_sample_by_the_recorded_run():
    """cost model: a Picard iteration costs (setup + GMRES iterations) units; the unit is the
    sample's median, so one slowed iteration does not move the estimate"""
    b = _bench()
    full = {"threads": 8, "picard_iterations": {"1e-06": 350, "0.0001": 180},
            "ksp_iterations": {"1e-06": 10000, "0.0001": 8000}, "setup_iterations": 10.0}
    sample = [(2.2, 100), (4.4, 100), (2.2, 100)]   # 20 ms per unit, the second iteration slowed
    est, how = b.cpu_estimate(0.5, sample, 1e-6, full=full)
    assert est == pytest.approx((0.5 + 0.02 * (10000 + 350 * 10.0)) * 1e3)
    assert "350 Picard" in how and "10000 GMRES" in how
    est4, _ = b.cpu_estimate(0.0, sample[:1], 1e-4, full=full)
    assert est4 == pytest.approx(0.02 * (8000 + 180 * 10.0) * 1e3)
    assert b.cpu_estimate(1.0, sample, 1e-7, full=full)[0] is None
    assert b.cpu_estimate(1.0, [], 1e-6, full=full)[0] is None


def test_recorded_run_predicts_itself():
    """the recorded complete 801^2 run's totals are consistent with its own cost model: a
    sample whose iterations cost exactly the model's unit reproduces n c + sum its"""
    b = _bench()
    full = b.CPU_FULL_RUN_801
    c = full["setup_iterations"]
    u = 0.05
    est, _ = b.cpu_estimate(0.0, [(u * (c + 221), 221), (u * (c + 223), 223)], 1e-6)
    assert est == pytest.approx(u * (full["ksp_iterations"]["1e-06"] + 359 * c) * 1e3)
    assert full["ksp_iterations"]["0.0001"] < full["ksp_iterations"]["1e-06"]
