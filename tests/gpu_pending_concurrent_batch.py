"""GPU test of pism_gpu_ssa_solve_batch_concurrent (members in flight on their own
streams through whole-solve graphs), not yet run on a GPU: this file is named outside
pytest's test_*.py pattern, so it is not collected until it has passed on a B200
(run it with  pytest -o python_files=gpu_pending_concurrent_batch.py <this file>).  The
bar: per member, bitwise the sequential batch's velocities and counts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200 import learned as Lr, synthetic as S  # noqa: E402
from pism_b200.ssa import SSAFD  # noqa: E402

NAMES = ("thickness", "surface", "bed", "mask", "tauc", "melange")


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
