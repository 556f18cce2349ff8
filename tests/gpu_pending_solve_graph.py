"""GPU tests of the whole-solve graph (graphs = 3) and of pism_gpu_ssa_solve_batch_concurrent.

Both modes are built but have not yet run on a GPU, so this file is named outside pytest's
test_*.py pattern and is not collected; it becomes tests/test_gpu_solve_graph.py once it
has passed on a B200.  The bar is the one the other launch modes meet: the same kernels in
the same order give bitwise the same velocities and the same counts.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200 import learned as Lr, synthetic as S  # noqa: E402
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


@pytest.mark.parametrize("pc,precision,adaptive", [("mg", "mixed", True), ("mg", "fp64", True),
                                                   ("mg", "fp64", False), ("bjacobi", "fp64", False),
                                                   ("line", "fp64", False)])
def test_whole_solve_graph_equals_graph_resident_loops(pc, precision, adaptive):
    g, c, f, _ = S.build_synthetic(41, 4000e3 / 40, seed=8)
    c = c.copy(pc_type=pc, precision=precision, ksp_rtol=1e-8, ksp_rtol_adaptive=adaptive, ksp_rtol_factor=1.0,
               ksp_rtol_max=1e-1)
    v2, s2 = solve(g, c.copy(graphs=2), f)
    v3, s3 = solve(g, c.copy(graphs=3), f)
    np.testing.assert_array_equal(v3, v2)
    for k in ("picard_iterations", "ksp_iterations", "refinement_steps", "converged", "strategy"):
        assert s3[k] == s2[k], k
    assert s3["final_linear_residual"] == s2["final_linear_residual"]
    assert s3["nuH_norm"] == s2["nuH_norm"] and s3["nuH_norm_change"] == s2["nuH_norm_change"]
    # the graph adds its control kernels: a few per Picard and refinement pass
    assert s2["kernel_launches"] < s3["kernel_launches"] < 1.3 * s2["kernel_launches"]


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


def ensemble(device, n=7, M=41):
    out = []
    rng = np.random.default_rng(3)
    for q in range(n):
        T, med = rng.uniform(-20, -2), rng.uniform(20e3, 200e3)
        g, c, f, _ = S.build_synthetic(M, 4000e3 / (M - 1), seed=40 + q, temperature_c=T, tauc_median=med)
        m = {k: (torch.tensor(f[k], device="cuda") if device else f[k]) for k in NAMES}
        m["ice_softness"] = c.ice_softness
        out.append(m)
    return g, c, out


@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("learned", [False, True])
def test_concurrent_batch_equals_sequential_batch(device, learned):
    g, c, mem = ensemble(device)
    cfg = c.copy(pc_type="mg", precision="mixed", ksp_rtol=1e-6, ksp_rtol_adaptive=True, ksp_rtol_factor=1.0,
                 ksp_rtol_max=1e-1)
    hh, ww = Lr.image_shape(41, 41, 1)
    net = Lr.UNet(1, hh, ww, params=np.load(Lr.DEFAULT_WEIGHTS)["params"]) if learned else None
    s = SSAFD(g, cfg)
    seq, st_seq = s.solve_batch([dict(m) for m in mem], net=net, stride=1)
    for streams in (3, 7):
        con, st_con = s.solve_batch([dict(m) for m in mem], net=net, stride=1, streams=streams)
        for q in range(len(mem)):
            a = con[q].cpu().numpy() if device else con[q]
            b = seq[q].cpu().numpy() if device else seq[q]
            np.testing.assert_array_equal(a, b)
            for k in ("status", "converged", "picard_iterations", "ksp_iterations", "refinement_steps"):
                assert st_con[q][k] == st_seq[q][k], (q, k)
    s.close()
