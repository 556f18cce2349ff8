"""The network oracle against finite differences (CPU): its backward pass is the gradient of
its forward pass, and its parameter layout is the one include/pism_unet_gpu.h declares."""
import os
import re

import numpy as np
import pytest

from oracle import unet_oracle as U

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_layout_matches_the_header():
    txt = open(os.path.join(REPO, "include", "pism_unet_gpu.h")).read()
    convs = re.findall(r"(\d+)->(\d+)", txt)
    assert [(int(a), int(b)) for a, b in convs] == [(c, o) for c, o, _ in U.LAYERS]
    assert U.param_count() == sum(9 * c * o + o for c, o, _ in U.LAYERS) + 2 * 32 + 2
    assert 550_000 < U.param_count() < 700_000


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 1e-30, 3.0e38], np.float32)
    r = U.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0   # tie -> even
    assert r[2] == np.float32(1.0 + 2 ** -7)
    assert r[3] == -2.5
    assert abs(r[4] - 1e-30) / 1e-30 < 2 ** -8


@pytest.mark.parametrize("seed", [0, 1])
def test_backward_is_the_gradient_of_forward(seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    p = U.init_params(seed).astype(np.float64)
    offs, head = U.layout()
    p[offs[0][1]:offs[0][1] + 32] = 0.05          # nonzero biases somewhere
    x = rng.standard_normal((1, 16, 16, 8))
    t = rng.standard_normal((1, 16, 16, 2))
    w = rng.uniform(0.5, 1.5, (1, 16, 16))
    net = U.UNetOracle(p, bf16=False)
    net.forward(x)
    loss, g = net.backward(t, w)
    idx = list(rng.choice(U.param_count(), 24, replace=False))
    idx += [head + k for k in (0, 33, 64, 65)] + [offs[0][0] + 5, offs[9][1] + 3, offs[6][0] + 1000]
    for k in idx:
        if offs[0][0] <= k < offs[0][1] and (k - offs[0][0]) % 16 >= 8:
            assert g[k] == 0.0          # padded input channels
            continue
        eps = 1e-6 * max(1.0, abs(p[k]))
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        a = U.UNetOracle(pp, bf16=False)
        a.forward(x)
        b = U.UNetOracle(pm, bf16=False)
        b.forward(x)
        fd = (a.loss(t, w) - b.loss(t, w)) / (2 * eps)
        assert fd == pytest.approx(g[k], rel=2e-4, abs=1e-9 * max(1.0, abs(loss))), k


def test_bf16_mode_tracks_float64():
    rng = np.random.Generator(np.random.PCG64(3))
    p = U.init_params(3)
    x = rng.standard_normal((2, 16, 24, 8)).astype(np.float32)
    t = rng.standard_normal((2, 16, 24, 2))
    lo, hi = U.UNetOracle(p, bf16=True), U.UNetOracle(p.astype(np.float64), bf16=False)
    ylo, yhi = lo.forward(x), hi.forward(x)
    assert np.linalg.norm(ylo - yhi) / np.linalg.norm(yhi) < 3e-2
    _, glo = lo.backward(t)
    _, ghi = hi.backward(t)
    assert np.linalg.norm(glo - ghi) / np.linalg.norm(ghi) < 5e-2
