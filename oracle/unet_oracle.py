"""CPU oracle of the learned warm start's network (test infrastructure only).

A numpy restatement of the U-Net declared in include/pism_unet_gpu.h: its forward pass, its
backward pass (the gradient of the weighted mean-square loss with respect to every
parameter) and the parameter layout.  With ``bf16=True`` it rounds to bfloat16 (round to
nearest even) at the same points as the CUDA kernels: the network input, the weights of the
convolutions, every stored activation and every stored activation gradient; sums are
formed in float64 and rounded to float32 where the GPU keeps FP32.  With ``bf16=False``
everything is float64, which the finite-difference check of the gradient uses.

No reference counterpart: PISM v0.7.3 has no learned component; the network only supplies
the initial velocity that SSA::set_initial_guess (src/base/stressbalance/ssa/SSA.cc:361-363)
would otherwise take from the previous step.
"""
from __future__ import annotations

import numpy as np

# (Cin, Cout, level) of the 10 convolutions, in parameter order
LAYERS = [(16, 32, 0), (32, 32, 0), (32, 64, 1), (64, 64, 1), (64, 96, 2),
          (96, 96, 2), (96, 128, 3), (224, 96, 2), (160, 64, 1), (96, 32, 0)]
HEAD_CIN, HEAD_COUT = 32, 2
IN_CHANNELS = 8


def layout():
    """[(w_offset, b_offset)] per convolution and the head's offset, in FP32 elements."""
    off, out = 0, []
    for cin, cout, _ in LAYERS:
        out.append((off, off + 9 * cout * cin))
        off += 9 * cout * cin + cout
    return out, off


def param_count():
    _, head = layout()
    return head + HEAD_COUT * HEAD_CIN + HEAD_COUT


def init_params(seed=0):
    """He-normal convolutions (fan-in of the real input channels), zero biases, a small head."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros(param_count(), np.float32)
    offs, head = layout()
    for (cin, cout, _), (wo, _bo) in zip(LAYERS, offs):
        real = IN_CHANNELS if cin == 16 else cin
        w = rng.standard_normal((9, cout, cin)).astype(np.float32) * np.float32(np.sqrt(2.0 / (9 * real)))
        if cin == 16:
            w[:, :, IN_CHANNELS:] = 0.0
        p[wo:wo + w.size] = w.ravel()
    p[head:head + HEAD_COUT * HEAD_CIN] = rng.standard_normal(HEAD_COUT * HEAD_CIN) * np.sqrt(1.0 / HEAD_CIN)
    return p


def bf16_round(x):
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


class UNetOracle:
    def __init__(self, params, bf16=True):
        self.bf16 = bf16
        self.p = np.asarray(params, np.float64 if not bf16 else np.float32).copy()
        self.offs, self.head = layout()

    # -- rounding helpers --
    def q(self, x):
        """a stored activation / activation gradient"""
        return bf16_round(np.asarray(x, np.float32)) if self.bf16 else np.asarray(x, np.float64)

    def f32(self, x):
        return np.asarray(x, np.float32) if self.bf16 else np.asarray(x, np.float64)

    def W(self, l):
        cin, cout, _ = LAYERS[l]
        wo, _ = self.offs[l]
        w = self.p[wo:wo + 9 * cout * cin].reshape(9, cout, cin)
        return bf16_round(w) if self.bf16 else w

    def b(self, l):
        cout = LAYERS[l][1]
        _, bo = self.offs[l]
        return self.p[bo:bo + cout]

    # -- primitives --
    @staticmethod
    def conv(x, w):
        """sum_tap x[p + (ky - 1, kx - 1)] . w[tap]^T with zero padding, in float64"""
        B, H, W, _ = x.shape
        xp = np.pad(np.asarray(x, np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
        out = np.zeros((B, H, W, w.shape[1]))
        for tap in range(9):
            ky, kx = divmod(tap, 3)
            out += xp[:, ky:ky + H, kx:kx + W, :] @ np.asarray(w[tap], np.float64).T
        return out

    @staticmethod
    def conv_back_data(dy, w):
        """dx[p] = sum_tap dy[p - (ky - 1, kx - 1)] . w[tap]"""
        B, H, W, _ = dy.shape
        dp = np.pad(np.asarray(dy, np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
        out = np.zeros((B, H, W, w.shape[2]))
        for tap in range(9):
            ky, kx = divmod(tap, 3)
            out += dp[:, 2 - ky:2 - ky + H, 2 - kx:2 - kx + W, :] @ np.asarray(w[tap], np.float64)
        return out

    @staticmethod
    def conv_back_weight(x, dy):
        """dw[tap] = sum_p dy[p]^T x[p + (ky - 1, kx - 1)]"""
        B, H, W, C = x.shape
        xp = np.pad(np.asarray(x, np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
        d = np.asarray(dy, np.float64).reshape(-1, dy.shape[-1])
        out = np.zeros((9, dy.shape[-1], C))
        for tap in range(9):
            ky, kx = divmod(tap, 3)
            out[tap] = d.T @ xp[:, ky:ky + H, kx:kx + W, :].reshape(-1, C)
        return out

    def pool(self, x):
        x = self.f32(x)
        s = x[:, 0::2, 0::2] + x[:, 0::2, 1::2]
        s = s + x[:, 1::2, 0::2]
        s = s + x[:, 1::2, 1::2]
        return self.q(s * self.f32(0.25))

    @staticmethod
    def up(x):
        return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)

    def layer(self, l, x):
        y = self.conv(x, self.W(l)) + np.asarray(self.b(l), np.float64)
        return self.q(np.maximum(self.f32(y), 0.0))

    # -- the network --
    def forward(self, inp):
        """inp [B, H, W, 8] -> y [B, H, W, 2]; keeps the activations for backward"""
        B, H, W, _ = inp.shape
        x16 = np.zeros((B, H, W, 16), np.float32 if self.bf16 else np.float64)
        x16[..., :IN_CHANNELS] = self.q(inp)
        a = {"in16": x16}
        a["e1a"] = self.layer(0, x16)
        a["e1"] = self.layer(1, a["e1a"])
        a["p1"] = self.pool(a["e1"])
        a["e2a"] = self.layer(2, a["p1"])
        a["e2"] = self.layer(3, a["e2a"])
        a["p2"] = self.pool(a["e2"])
        a["e3a"] = self.layer(4, a["p2"])
        a["e3"] = self.layer(5, a["e3a"])
        a["p3"] = self.pool(a["e3"])
        a["bt"] = self.layer(6, a["p3"])
        a["c3"] = np.concatenate([self.up(a["bt"]), a["e3"]], axis=-1)
        a["d3"] = self.layer(7, a["c3"])
        a["c2"] = np.concatenate([self.up(a["d3"]), a["e2"]], axis=-1)
        a["d2"] = self.layer(8, a["c2"])
        a["c1"] = np.concatenate([self.up(a["d2"]), a["e1"]], axis=-1)
        a["d1"] = self.layer(9, a["c1"])
        wh = self.p[self.head:self.head + HEAD_COUT * HEAD_CIN].reshape(HEAD_COUT, HEAD_CIN)
        bh = self.p[self.head + HEAD_COUT * HEAD_CIN:]
        y = np.asarray(a["d1"], np.float64) @ np.asarray(wh, np.float64).T + bh
        a["y"] = self.f32(y)
        self.a = a
        return a["y"]

    def loss(self, target, weight=None):
        y = np.asarray(self.a["y"], np.float64)
        w = np.ones(y.shape[:-1]) if weight is None else np.asarray(weight, np.float64)
        return float((w[..., None] * (y - target) ** 2).sum() / (2.0 * w.sum()))

    def backward(self, target, weight=None):
        """(loss, gradient [param_count]) of the last forward"""
        a = self.a
        y = np.asarray(a["y"], np.float64)
        w = np.ones(y.shape[:-1]) if weight is None else np.asarray(weight, np.float64)
        g = np.zeros(param_count())
        e = self.f32(w[..., None] * (y - target) / w.sum())
        wh = self.p[self.head:self.head + HEAD_COUT * HEAD_CIN].reshape(HEAD_COUT, HEAD_CIN)
        d1 = np.asarray(a["d1"], np.float64)
        g[self.head:self.head + HEAD_COUT * HEAD_CIN] = (np.asarray(e, np.float64).reshape(-1, 2).T
                                                        @ d1.reshape(-1, HEAD_CIN)).ravel()
        g[self.head + HEAD_COUT * HEAD_CIN:] = np.asarray(e, np.float64).reshape(-1, 2).sum(axis=0)
        dd1 = self.q(np.asarray(e, np.float64) @ np.asarray(wh, np.float64))

        def back(l, x, yl, dy, need_dx=True):
            dpre = np.where(np.asarray(yl) > 0, dy, 0.0)
            wo, bo = self.offs[l]
            cin, cout, _ = LAYERS[l]
            g[wo:wo + 9 * cout * cin] = self.conv_back_weight(x, dpre).ravel()
            g[bo:bo + cout] = np.asarray(dpre, np.float64).reshape(-1, cout).sum(axis=0)
            return self.q(self.conv_back_data(dpre, self.W(l))) if need_dx else None

        def upcat_back(dc, cu):
            du = self.f32(dc[..., :cu])
            s = du[:, 0::2, 0::2] + du[:, 0::2, 1::2]
            s = s + du[:, 1::2, 0::2]
            s = s + du[:, 1::2, 1::2]
            return self.q(s), dc[..., cu:].copy()

        def pool_back_add(dx, dp):
            return self.q(self.f32(dx) + self.f32(0.25) * self.f32(self.up(dp)))

        dc1 = back(9, a["c1"], a["d1"], dd1)
        dd2, de1 = upcat_back(dc1, 64)
        dc2 = back(8, a["c2"], a["d2"], dd2)
        dd3, de2 = upcat_back(dc2, 96)
        dc3 = back(7, a["c3"], a["d3"], dd3)
        dbt, de3 = upcat_back(dc3, 128)
        dp3 = back(6, a["p3"], a["bt"], dbt)
        de3 = pool_back_add(de3, dp3)
        de3a = back(5, a["e3a"], a["e3"], de3)
        dp2 = back(4, a["p2"], a["e3a"], de3a)
        de2 = pool_back_add(de2, dp2)
        de2a = back(3, a["e2a"], a["e2"], de2)
        dp1 = back(2, a["p1"], a["e2a"], de2a)
        de1 = pool_back_add(de1, dp1)
        de1a = back(1, a["e1a"], a["e1"], de1)
        back(0, a["in16"], a["e1a"], de1a, need_dx=False)
        return self.loss(target, weight), g


def velocity_transform(u_mps, secpera=31556925.9747):
    """the network's target: asinh(u / (10 m/yr)) per component"""
    return np.arcsinh(np.asarray(u_mps) * secpera / 10.0)


def velocity_from_output(y, secpera=31556925.9747):
    return 10.0 * np.sinh(np.asarray(y, np.float64)) / secpera
