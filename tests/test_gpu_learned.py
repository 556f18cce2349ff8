"""What the trained warm-start network gains: on sheets it was not trained on, the solve
from its prediction needs far fewer Picard iterations than the same solve from zero, and
meets the same stopping tests (Picard nu*H change, final linear residual)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200 import learned as Lr  # noqa: E402
from pism_b200.ssa import SSAFD  # noqa: E402

NAMES = ("thickness", "surface", "bed", "mask", "tauc", "melange")


def fast(c):
    return c.copy(pc_type="mg", precision="mixed", ksp_rtol=1e-6, ksp_rtol_adaptive=True, ksp_rtol_factor=0.1,
                  ksp_rtol_max=1e-2)


@pytest.mark.skipif(not os.path.exists(Lr.DEFAULT_WEIGHTS), reason="no trained weights")
@pytest.mark.parametrize("seed", [5000, 5001])   # training used seeds below 1024
def test_learned_guess_cuts_picard_iterations(seed):
    g, c, f, _ = Lr.training_case(seed, 401)
    hh, ww = Lr.image_shape(401, 401, 1)
    net = Lr.UNet(1, hh, ww, params=np.load(Lr.DEFAULT_WEIGHTS)["params"])
    res = {}
    for mode in ("zero", "learned"):
        s = SSAFD(g, fast(c))
        s.set_inputs(**{k: f[k] for k in NAMES})
        if mode == "learned":
            Lr.learned_guess(s, net, 1)
            guess = s.velocity()
            assert np.all(np.isfinite(guess)) and np.abs(guess).max() > 0
        res[mode] = (s.solve(), s.stats())
        s.close()
    net.close()
    (u0, st0), (u1, st1) = res["zero"], res["learned"]
    for st in (st0, st1):
        assert st["converged"] == 1 and st["final_linear_residual"] <= 1e-6
        assert st["nuH_norm_change"] / st["nuH_norm"] < c.ssafd_relative_convergence
    assert st1["picard_iterations"] < 0.75 * st0["picard_iterations"], (st1["picard_iterations"],
                                                                         st0["picard_iterations"])
    # both answers stop within the Picard tolerance of the same fixed point
    assert np.linalg.norm(u1 - u0) / np.linalg.norm(u0) < 2e-2
