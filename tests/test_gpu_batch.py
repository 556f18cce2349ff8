"""pism_gpu_ssa_solve_batch: an ensemble of independent sheets on one handle gives, member
by member, exactly what separate solves give (same kernels, same order), with and without
the learned initial guess, and reports per-member statistics."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200 import _capi, learned as Lr, synthetic as S  # noqa: E402
from pism_b200.config import CMember, CStats  # noqa: E402
from pism_b200.ssa import SSAFD  # noqa: E402

NAMES = ("thickness", "surface", "bed", "mask", "tauc", "melange")
M = 41


def members(device):
    out = []
    for q, (T, med) in enumerate(((-10.0, 50e3), (-3.0, 30e3), (-18.0, 150e3))):
        g, c, f, _ = S.build_synthetic(M, 4000e3 / (M - 1), seed=20 + q, temperature_c=T, tauc_median=med)
        m = {k: (torch.tensor(f[k], device="cuda") if device else f[k]) for k in NAMES}
        m["ice_softness"] = c.ice_softness
        out.append(m)
    return g, c, out


def config(c):
    return c.copy(pc_type="mg", precision="mixed", ksp_rtol=1e-6, ksp_rtol_adaptive=True, ksp_rtol_factor=0.1,
                  ksp_rtol_max=1e-2)


@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("learned", [False, True])
def test_batch_equals_separate_solves(device, learned):
    g, c, mem = members(device)
    cfg = config(c)
    hh, ww = Lr.image_shape(M, M, 1)
    net = Lr.UNet(1, hh, ww, params=np.load(Lr.DEFAULT_WEIGHTS)["params"]) if learned else None
    s = SSAFD(g, cfg)
    vels, stats = s.solve_batch(mem, net=net, stride=1)
    s.close()
    for q, m in enumerate(mem):
        one = SSAFD(g, cfg.copy(ice_softness=m["ice_softness"]))
        one.set_inputs(**{k: m[k] for k in NAMES})
        if learned:
            Lr.learned_guess(one, net, 1)
        ref = one.solve()
        st = one.stats()
        one.close()
        got = vels[q].cpu().numpy() if device else vels[q]
        np.testing.assert_array_equal(got, ref)
        assert stats[q]["status"] == 0 and stats[q]["converged"] == 1
        assert stats[q]["picard_iterations"] == st["picard_iterations"]
        assert stats[q]["ksp_iterations"] == st["ksp_iterations"]
    if net is not None:
        net.close()


def test_batch_rejects_a_member_without_velocity():
    g, c, mem = members(False)
    s = SSAFD(g, config(c))
    ci, keep = s._inputs({k: mem[0][k] for k in NAMES} | {"gl_mask": None, "enthalpy": None, "hardness": None,
                                                           "fracture_density": None}, (None, None))
    arr = (CMember * 1)()
    arr[0].inputs = ci
    arr[0].velocity = None
    st = (CStats * 1)()
    assert s.lib.pism_gpu_ssa_solve_batch(s._h, None, 1, 1, arr, st) == _capi.EINVAL
    s.close()
