"""The warm-start network's CUDA kernels against the CPU oracle (oracle/unet_oracle.py):
forward output, loss, every parameter gradient and the Adam step; the feature image and the
learned guess against their definitions in include/pism_unet_gpu.h.

Tolerances: the GPU and the oracle round to bfloat16 at the same points but sum in a
different order, so an occasional stored value differs by one bfloat16 ulp (2^-8) and
the difference propagates through up to 16 rounded stages of the backward pass: outputs
agree to 1e-2, each layer's gradient to 6e-2 relative L2 (3e-2 on average over the
layers).  The oracle's bfloat16 mode itself moves the gradients by a few per cent from
its float64 mode, which finite differences pin (tests/test_unet_oracle.py); a layout or
indexing error shows up as an O(1) difference."""
import numpy as np
import pytest

from oracle import unet_oracle as U

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200 import learned as Lr, synthetic as S  # noqa: E402
from pism_b200.ssa import SSAFD  # noqa: E402

DEV = torch.device("cuda", 0)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def params(seed):
    p = U.init_params(seed)
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    offs, head = U.layout()
    for (cin, cout, _), (wo, bo) in zip(U.LAYERS, offs):
        p[bo:bo + cout] = rng.normal(0, 0.05, cout)
    p[head + 64:] = [0.1, -0.2]
    return p


@pytest.mark.parametrize("B,H,W", [(1, 16, 16), (2, 16, 24), (1, 32, 40)])
def test_forward_backward_match_the_oracle(B, H, W):
    rng = np.random.Generator(np.random.PCG64(B * 100 + H + W))
    p = params(B + H)
    x = rng.standard_normal((B, H, W, 8)).astype(np.float32)
    t = rng.standard_normal((B, H, W, 2)).astype(np.float32)
    w = rng.uniform(0.2, 1.0, (B, H, W)).astype(np.float32)
    o = U.UNetOracle(p, bf16=True)
    y_ref = o.forward(x)
    loss_ref, g_ref = o.backward(t, w)

    net = Lr.UNet(B, H, W, params=p)
    y = net.forward(torch.tensor(x, device=DEV)).cpu().numpy()
    g = torch.empty(U.param_count(), dtype=torch.float32, device=DEV)
    loss = net.backward(torch.tensor(t, device=DEV), torch.tensor(w, device=DEV), grad_out=g)
    g = g.cpu().numpy()
    net.close()
    assert rel(y, y_ref) < 1e-2
    assert loss == pytest.approx(loss_ref, rel=2e-2)
    offs, head = U.layout()
    errs = []
    for l, ((cin, cout, _), (wo, bo)) in enumerate(zip(U.LAYERS, offs)):
        errs += [rel(g[wo:bo], g_ref[wo:bo]), rel(g[bo:bo + cout], g_ref[bo:bo + cout])]
    assert max(errs) < 6e-2 and np.mean(errs) < 3e-2, np.round(errs, 4)
    assert rel(g[head:], g_ref[head:]) < 1e-2
    # padded input channels get no gradient
    w0 = g[offs[0][0]:offs[0][1]].reshape(9, 32, 16)
    assert np.all(w0[:, :, 8:] == 0)


def test_adam_step_matches_numpy():
    rng = np.random.Generator(np.random.PCG64(5))
    p = params(3)
    x = torch.tensor(rng.standard_normal((1, 16, 16, 8)).astype(np.float32), device=DEV)
    t = torch.tensor(rng.standard_normal((1, 16, 16, 2)).astype(np.float32), device=DEV)
    net = Lr.UNet(1, 16, 16, params=p)
    g = torch.empty(U.param_count(), dtype=torch.float32, device=DEV)
    m = np.zeros(p.size)
    v = np.zeros(p.size)
    q = p.astype(np.float64)
    for step in (1, 2):
        net.forward(x)
        net.backward(t, grad_out=g)
        gn = g.cpu().numpy().astype(np.float64)
        net.adam(1e-3, 0.9, 0.999, 1e-8)
        m = 0.9 * m + 0.1 * gn
        v = 0.999 * v + 0.001 * gn * gn
        q = q - 1e-3 * (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8)
        got = net.get_params()
        assert np.max(np.abs(got - q)) < 1e-6
        x = x * 1.01
    net.close()


@pytest.mark.parametrize("augment", [False, True])
def test_training_lowers_the_loss(augment):
    """A pointwise target of the inputs is learned in a few hundred steps (an FP32 PyTorch
    model of the same network and schedule goes from 0.54 to 0.05 on the first target).
    The second target has the SSA's mirror / transpose symmetry, which the augmentation
    assumes: u and tau_d x reverse under a flip of the first axis, and so on."""
    rng = np.random.Generator(np.random.PCG64(11))
    xs = torch.tensor(rng.standard_normal((64, 32, 32, 8)).astype(np.float32), device=DEV)
    if augment:
        amp = 1.0 + 0.5 * torch.tanh(xs[..., 0])
        ts = torch.stack([xs[..., 6] * amp, xs[..., 7] * amp], dim=-1)
    else:
        ts = torch.stack([torch.tanh(xs[..., 0] + 0.5 * xs[..., 1]), 0.3 * xs[..., 2] * xs[..., 3]], dim=-1)
    data = [(xs[k], ts[k].contiguous(), torch.ones((32, 32), device=DEV)) for k in range(64)]
    net = Lr.UNet(8, 32, 32, seed=1)
    before = Lr.evaluate(net, data[:8])
    Lr.train(net, data, steps=300, batch=8, crop=32, lr=2e-3, warmup=20, seed=0, augment=augment)
    after = Lr.evaluate(net, data[:8])
    net.close()
    assert after < 0.3 * before


def test_features_and_guess_follow_their_definition():
    M = 37
    g, c, f, _ = S.build_synthetic(M, 4000e3 / (M - 1), seed=4)
    s = SSAFD(g, c)
    s.set_inputs(**{k: f[k] for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")})
    for stride in (1, 2):
        x = Lr.features(s, stride).cpu().numpy()
        taud = s.driving_stress()
        hard = s.hardness()
        sl = (slice(0, M, stride), slice(0, M, stride))
        n = -(-M // stride)
        assert x.shape == (*Lr.image_shape(M, M, stride), 8)
        mask = f["mask"][sl]
        icy = (mask == 2) | (mask == 3)
        np.testing.assert_allclose(x[:n, :n, 0], f["thickness"][sl] * 1e-3, rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(x[:n, :n, 1], f["bed"][sl] * 1e-3, rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(x[:n, :n, 2], np.log(np.maximum(f["tauc"][sl], 1.0) / 5e4), rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(x[:n, :n, 3], np.where(icy, hard[sl].max(axis=-1) * 1e-8, 0), rtol=1e-6)
        np.testing.assert_array_equal(x[:n, :n, 4], (mask == 2).astype(np.float32))
        np.testing.assert_array_equal(x[:n, :n, 5], (mask == 3).astype(np.float32))
        np.testing.assert_allclose(x[:n, :n, 6:], taud[sl] * 1e-5, rtol=1e-6, atol=1e-9)
        assert np.all(x[n:] == 0) and np.all(x[:, n:] == 0)
    # a network whose output is the constant (asinh 1, asinh 2): 10 and 20 m/yr everywhere
    p = np.zeros(U.param_count(), np.float32)
    p[-2:] = [np.arcsinh(1.0), np.arcsinh(2.0)]
    hh, ww = Lr.image_shape(M, M, 2)
    net = Lr.UNet(1, hh, ww, params=p)
    Lr.learned_guess(s, net, 2)
    vel = s.velocity() * Lr.SECPERA
    np.testing.assert_allclose(vel[..., 0], 10.0, rtol=1e-6)
    np.testing.assert_allclose(vel[..., 1], 20.0, rtol=1e-6)
    net.close()
    s.close()
