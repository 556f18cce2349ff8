"""The whole-solve graph (graphs = 3): the Picard loop of a solve as one CUDA graph with
nested conditional nodes, its decisions taken on the device.  The same kernels in the same
order as graphs = 2 give bitwise the same velocities and the same counts, for the mixed and
the FP64 set-ups with each preconditioner; a zero diagonal and a KSP failure come out as
with the host loop (the failure then goes through the host's fallback ladder)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200 import synthetic as S  # noqa: E402
from pism_b200.ssa import SSAFD, KSPFailure, ZeroDiagonal  # noqa: E402
from pism_b200.config import SSAConfig, GridDesc  # noqa: E402

NAMES = ("thickness", "surface", "bed", "mask", "tauc", "melange")


def solve(g, c, f):
    s = SSAFD(g, c)
    s.set_inputs(**{k: f[k] for k in NAMES})
    vel = s.solve()
    st = s.stats()
    s.close()
    return vel, st


@pytest.mark.parametrize("pc,precision,adaptive,lag", [("mg", "mixed", True, 0.0), ("mg", "fp64", True, 0.0),
                                                       ("mg", "fp64", False, 0.0), ("bjacobi", "fp64", False, 0.0),
                                                       ("line", "fp64", False, 0.0), ("mg", "mixed", True, 0.05),
                                                       ("mg", "fp64", False, 0.05)])
def test_whole_solve_graph_equals_graph_resident_loops(pc, precision, adaptive, lag):
    """lag > 0: lagged multigrid coarse levels (the graph's IF node around the coarse
    build against the host loop's decision)"""
    g, c, f, _ = S.build_synthetic(41, 4000e3 / 40, seed=8)
    c = c.copy(pc_type=pc, precision=precision, ksp_rtol=1e-8, ksp_rtol_adaptive=adaptive, ksp_rtol_factor=1.0,
               ksp_rtol_max=1e-1, mg_rebuild_rtol=lag)
    v2, s2 = solve(g, c.copy(graphs=2), f)
    v3, s3 = solve(g, c.copy(graphs=3), f)
    np.testing.assert_array_equal(v3, v2)
    for k in ("picard_iterations", "ksp_iterations", "refinement_steps", "converged", "strategy", "mg_rebuilds"):
        assert s3[k] == s2[k], k
    if lag > 0:
        assert 1 <= s2["mg_rebuilds"] < s2["picard_iterations"]
    elif pc == "mg":
        assert s2["mg_rebuilds"] == s2["picard_iterations"]
    assert s3["final_linear_residual"] == s2["final_linear_residual"]
    assert s3["nuH_norm"] == s2["nuH_norm"] and s3["nuH_norm_change"] == s2["nuH_norm_change"]
    # the graph adds its single-thread control kernels: about six per Picard pass and three
    # per refinement step (+37 % on this 41^2 sheet with the mixed set-up)
    assert s2["kernel_launches"] < s3["kernel_launches"] < 2.0 * s2["kernel_launches"]


def test_whole_solve_graph_reports_a_zero_diagonal():
    """The device-side check gives the host loop's error (SSAFD.cc:766-776)."""
    M = 9
    g = GridDesc(M, M, 40e3, 40e3, periodicity=0)
    c = SSAConfig(flow_law="isothermal_glen", graphs=3)
    f = {"thickness": np.zeros((M, M)), "surface": np.zeros((M, M)), "bed": np.full((M, M), -500.0),
         "mask": np.full((M, M), 4.0), "tauc": np.zeros((M, M)), "melange": np.zeros((M, M))}
    c.constant_nu_strength_extension_ssa = 0.0
    c.epsilon_ssa = 0.0
    s = SSAFD(g, c)
    s.set_inputs(**f)
    with pytest.raises(ZeroDiagonal):
        s.solve()
    s.close()


def test_whole_solve_graph_ksp_failure_goes_to_the_host_ladder():
    """A KSP failure inside the graph: the host's fallback and report, as with graphs = 2."""
    g, c, f, _ = S.build_synthetic(41, 4000e3 / 40, seed=9)
    c = c.copy(pc_type="mg", precision="fp64", ksp_rtol=1e-10, ksp_max_it=2, graphs=3)
    s = SSAFD(g, c)
    s.set_inputs(**{k: f[k] for k in NAMES})
    with pytest.raises(KSPFailure):
        s.solve()
    s.set_config(c.copy(ksp_max_it=10000))
    s.set_initial_guess(np.zeros((g.Mx, g.My, 2)))
    vel = s.solve()
    assert s.stats()["converged"] == 1 and np.all(np.isfinite(vel))
    s.close()
