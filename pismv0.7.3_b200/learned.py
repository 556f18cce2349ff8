"""The learned warm start of the SSA solve.

* ``UNet``: the network of include/pism_unet_gpu.h (BF16, hand-written CUDA forward,
  backward and Adam kernels in csrc/unet.cu) behind its C-ABI;
* ``features`` / ``learned_guess``: the network's input image built on the device from an
  SSAFD handle, and the initial velocity it predicts (pism_gpu_ssa_learned_guess);
* ``generate`` / ``train``: training data from solves of the plain solver (seeded synthetic
  ice sheets) and the training loop (random crops, flips and transposes, weighted MSE on
  asinh(u / 10 m/yr)).

The solver decides what is accepted: a learned guess only replaces the zero / previous-step initial
velocity of SSA::set_initial_guess (src/base/stressbalance/ssa/SSA.cc:361-363); the Picard
and Krylov stopping tests are unchanged.  There is no CPU fallback: without the compiled
library every call raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time

import numpy as np

from . import _capi
from . import synthetic as S
from .config import SSAConfig

SECPERA = 31556925.9747
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "unet_ssa_10km.npz")
IN_CHANNELS, OUT_CHANNELS = 8, 2


class UNetError(RuntimeError):
    pass


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class UNet:
    """The warm-start network on one device (images up to max_batch x max_h x max_w)."""

    def __init__(self, max_batch: int, max_h: int, max_w: int, device: int = 0, params=None, seed: int = 0):
        self.lib = _capi.load()
        self._h = C.c_void_p()
        rc = self.lib.pism_gpu_unet_create(device, max_batch, max_h, max_w, C.byref(self._h))
        if rc != _capi.OK:
            raise UNetError(f"pism_gpu_unet_create({device}, {max_batch}, {max_h}, {max_w}) failed (status {rc})")
        self.device = device
        self.shape = (max_batch, max_h, max_w)
        if params is None:
            params = init_params(seed)
        self.set_params(params)

    @staticmethod
    def param_count() -> int:
        return int(_capi.load().pism_gpu_unet_param_count())

    def _check(self, rc, what):
        if rc != _capi.OK:
            raise UNetError(f"{what}: {self.lib.pism_gpu_unet_last_error(self._h).decode()} (status {rc})")

    def close(self):
        if self._h:
            self.lib.pism_gpu_unet_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, cuda_stream_ptr):
        self._check(self.lib.pism_gpu_unet_set_stream(self._h, C.c_void_p(cuda_stream_ptr or 0)), "set_stream")

    def set_params(self, params):
        p = np.ascontiguousarray(np.asarray(params, np.float32))
        if p.size != self.param_count():
            raise UNetError(f"expected {self.param_count()} parameters, got {p.size}")
        self._check(self.lib.pism_gpu_unet_set_params(self._h, p.ctypes.data_as(C.c_void_p), _capi.MEM_HOST),
                    "set_params")

    def get_params(self) -> np.ndarray:
        p = np.empty(self.param_count(), np.float32)
        self._check(self.lib.pism_gpu_unet_get_params(self._h, p.ctypes.data_as(C.c_void_p), _capi.MEM_HOST),
                    "get_params")
        return p

    def forward(self, x, out=None):
        """x: CUDA float32 [B, H, W, 8] -> CUDA float32 [B, H, W, 2]"""
        import torch
        x = x.contiguous()
        B, H, W, _ = x.shape
        if out is None:
            out = torch.empty((B, H, W, OUT_CHANNELS), dtype=torch.float32, device=x.device)
        self._check(self.lib.pism_gpu_unet_forward(self._h, _ptr(x), B, H, W, _ptr(out)), "forward")
        return out

    def backward(self, target, weight=None, grad_out=None) -> float:
        """weighted MSE of the last forward against target ([B, H, W, 2]); returns the loss"""
        loss = C.c_float(0.0)
        t = target.contiguous()
        w = weight.contiguous() if weight is not None else None
        self._check(self.lib.pism_gpu_unet_backward(self._h, _ptr(t), _ptr(w) if w is not None else None,
                                                    C.byref(loss), _ptr(grad_out) if grad_out is not None else None),
                    "backward")
        return loss.value

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        self._check(self.lib.pism_gpu_unet_adam(self._h, lr, beta1, beta2, eps), "adam")

    def save(self, path: str, **meta):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, params=self.get_params(), **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, max_batch=1, max_h=408, max_w=408, device=0):
        d = np.load(path)
        return cls(max_batch, max_h, max_w, device=device, params=d["params"])


def init_params(seed: int) -> np.ndarray:
    """He-normal convolutions over the real fan-in, zero biases, a small head (the layout
    of include/pism_unet_gpu.h)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    layers = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 96), (96, 96), (96, 128), (224, 96), (160, 64), (96, 32)]
    out = []
    for cin, cout in layers:
        real = IN_CHANNELS if cin == 16 else cin
        w = rng.standard_normal((9, cout, cin)).astype(np.float32) * np.float32(math.sqrt(2.0 / (9 * real)))
        if cin == 16:
            w[:, :, IN_CHANNELS:] = 0.0
        out += [w.ravel(), np.zeros(cout, np.float32)]
    out += [(rng.standard_normal(64) * math.sqrt(1.0 / 32)).astype(np.float32), np.zeros(2, np.float32)]
    return np.concatenate(out)


# ---------------------------------------------------------------------------
# features and the learned guess
# ---------------------------------------------------------------------------
def image_shape(Mx: int, My: int, stride: int):
    return (-(-Mx // stride) + 7) // 8 * 8, (-(-My // stride) + 7) // 8 * 8


def features(ssa, stride: int = 1):
    """the network's input image of an SSAFD handle (inputs set): CUDA float32 [H8, W8, 8]"""
    import torch
    hh, ww = image_shape(*ssa.shape, stride)
    f = torch.empty((hh, ww, IN_CHANNELS), dtype=torch.float32, device=torch.device("cuda", ssa.device))
    ssa._check(ssa.lib.pism_gpu_ssa_learned_features(ssa._h, stride, _ptr(f), hh, ww), "learned_features")
    return f


def learned_guess(ssa, net: UNet, stride: int = 1):
    """replace the handle's initial guess by the network's prediction"""
    ssa._check(ssa.lib.pism_gpu_ssa_learned_guess(ssa._h, net._h, stride), "learned_guess")


def target_image(vel, hh, ww):
    """asinh(u / 10 m/yr) of a velocity [Mx, My, 2] (m/s), zero-padded to [hh, ww, 2]"""
    import torch
    Mx, My, _ = vel.shape
    t = torch.zeros((hh, ww, 2), dtype=torch.float32, device=vel.device)
    t[:Mx, :My] = torch.asinh(vel * (SECPERA / 10.0)).float()
    return t


# ---------------------------------------------------------------------------
# training data and training
# ---------------------------------------------------------------------------
def training_case(seed: int, M: int = 401, domain: float = 4000e3):
    """A seeded synthetic sheet for training: even seeds use the 801^2 benchmark's
    distribution (-10 C, tau_c median 50 kPa); odd seeds draw the ice temperature from
    U[-20, -2] C and the tau_c median from U[20, 200] kPa (the ensemble's ranges)."""
    rng = np.random.Generator(np.random.PCG64(10_000 + seed))
    if seed % 2 == 0:
        T, med = -10.0, 50e3
    else:
        T, med = rng.uniform(-20.0, -2.0), rng.uniform(20e3, 200e3)
    return S.build_synthetic(M, domain / (M - 1), seed=100_000 + seed, temperature_c=T, tauc_median=med)


def solve_config(c: SSAConfig) -> SSAConfig:
    """the plain solver's FP64 Picard / BiCGStab + multigrid path; the early Picard
    iterations' linear solves are inexact, the accepted one meets KSP rtol 1e-8"""
    return c.copy(pc_type="mg", precision="fp64", ksp_rtol=1e-8, ksp_rtol_adaptive=True, ksp_rtol_factor=0.1,
                  ksp_rtol_max=1e-2, ssafd_relative_convergence=1e-4)


def generate(seeds, M: int = 401, device: int = 0, log=None):
    """Solve the training cases one after another on one solver handle and return
    [(features [H8, W8, 8], target [H8, W8, 2], weight [H8, W8])] on the device plus per-case
    stats.  The handle's work runs on a stream of its own; every output is complete on
    return."""
    import torch
    from .ssa import SSAFD
    dev = torch.device("cuda", device)
    out = [None] * len(seeds)
    stats = [None] * len(seeds)
    stream = torch.cuda.Stream(device=dev)
    s = None
    try:
        with torch.cuda.stream(stream):
            for q, seed in enumerate(seeds):
                g, c, f, meta = training_case(seed, M)
                if s is None:
                    s = SSAFD(g, solve_config(c), device=device)
                    s.set_stream(stream.cuda_stream)
                else:
                    s.set_config(solve_config(c))
                s.set_inputs(**{k: f[k] for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")})
                vel = torch.empty((M, M, 2), dtype=torch.float64, device=dev)
                s.set_initial_guess(torch.zeros_like(vel))
                s.solve(out=vel)
                st = s.stats()
                x = features(s, 1)
                hh, ww = x.shape[:2]
                t = target_image(vel, hh, ww)
                m = torch.zeros((hh, ww), dtype=torch.float32, device=dev)
                mask = torch.tensor(f["mask"], device=dev)
                m[:M, :M] = torch.where((mask == 2) | (mask == 3), 1.0, 0.2).float()
                out[q] = (x, t, m)
                stats[q] = {"seed": seed, "picard": st["picard_iterations"], "ksp": st["ksp_iterations"],
                            "converged": st["converged"], "ms": st["kernel_ms"]}
                if log:
                    log(f"case {q} seed {seed}: {st['picard_iterations']} Picard, {st['kernel_ms']:.0f} ms")
        stream.synchronize()
    finally:
        if s is not None:
            s.close()
    return out, stats


def _augment(x, t, w, k):
    """flip along the first axis (u, tau_d x change sign), the second (v, tau_d y) and
    transpose (swap the components) as the bits of k say"""
    if k & 1:
        x, t, w = x.flip(0).clone(), t.flip(0).clone(), w.flip(0)
        x[..., 6] = -x[..., 6]
        t[..., 0] = -t[..., 0]
    if k & 2:
        x, t, w = x.flip(1).clone(), t.flip(1).clone(), w.flip(1)
        x[..., 7] = -x[..., 7]
        t[..., 1] = -t[..., 1]
    if k & 4:
        x = x.transpose(0, 1)[..., [0, 1, 2, 3, 4, 5, 7, 6]]
        t = t.transpose(0, 1)[..., [1, 0]]
        w = w.transpose(0, 1)
    return x, t, w


def sample_batch(data, batch: int, crop: int, rng, augment: bool = True):
    """random crops (centred on ice with probability 3/4) with random flips / transposes
    (the symmetries of the SSA: mirroring an axis reverses that velocity component and
    that driving-stress component)"""
    import torch
    xs, ts, ws = [], [], []
    for _ in range(batch):
        x, t, w = data[int(rng.integers(len(data)))]
        hh, ww = x.shape[:2]
        if rng.random() < 0.75:
            icy = (x[..., 4] + x[..., 5]) > 0
            idx = torch.nonzero(icy)
            c = idx[int(rng.integers(len(idx)))].tolist() if len(idx) else [hh // 2, ww // 2]
            i0 = int(np.clip(c[0] - crop // 2 + rng.integers(-crop // 4, crop // 4 + 1), 0, hh - crop))
            j0 = int(np.clip(c[1] - crop // 2 + rng.integers(-crop // 4, crop // 4 + 1), 0, ww - crop))
        else:
            i0, j0 = int(rng.integers(hh - crop + 1)), int(rng.integers(ww - crop + 1))
        a = _augment(x[i0:i0 + crop, j0:j0 + crop], t[i0:i0 + crop, j0:j0 + crop], w[i0:i0 + crop, j0:j0 + crop],
                     int(rng.integers(8)) if augment else 0)
        xs.append(a[0])
        ts.append(a[1])
        ws.append(a[2])
    return torch.stack(xs).contiguous(), torch.stack(ts).contiguous(), torch.stack(ws).contiguous()


def train(net: UNet, data, steps: int, batch: int = 16, crop: int = 128, lr: float = 2e-3, lr_min: float = 2e-5,
          warmup: int = 100, seed: int = 0, log=None, log_every: int = 100, augment: bool = True):
    """Adam with linear warm-up and cosine decay; returns the loss history"""
    rng = np.random.Generator(np.random.PCG64(seed))
    hist = []
    t0 = time.perf_counter()
    for k in range(steps):
        x, t, w = sample_batch(data, batch, crop, rng, augment)
        net.forward(x)
        loss = net.backward(t, w)
        if not math.isfinite(loss):
            raise UNetError(f"non-finite training loss at step {k}")
        a = min(1.0, (k + 1) / warmup)
        rate = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * k / max(1, steps - 1)))
        net.adam(a * rate)
        hist.append(loss)
        if log and (k % log_every == 0 or k == steps - 1):
            log(f"step {k}: loss {np.mean(hist[-log_every:]):.5f} ({time.perf_counter() - t0:.1f} s)")
    return hist


def evaluate(net: UNet, data):
    """mean weighted MSE of whole images (batch 1, no augmentation)"""
    out = []
    for x, t, w in data:
        net.forward(x[None].contiguous())
        out.append(net.backward(t[None].contiguous(), w[None].contiguous()))
    return float(np.mean(out))


# ---------------------------------------------------------------------------
# the learned preconditioner correction inside flexible GMRES
# ---------------------------------------------------------------------------
PC_WEIGHTS = os.path.join(WEIGHTS_DIR, "unet_ssa_pc_10km.npz")


def set_learned_pc(ssa, net, stride: int = 1):
    """attach the correction network to the handle's GMRES solves (net None detaches it)"""
    ssa._check(ssa.lib.pism_gpu_ssa_set_learned_pc(ssa._h, net._h if net is not None else None, stride),
               "set_learned_pc")


def pc_input(ssa, r, stride: int = 1):
    """the correction network's input for a residual r (CUDA float64 [Mx, My, 2]) at the
    handle's current nu*H and beta: (image [H8, W8, 8] float32, rho as a 0-d float64 tensor)"""
    import torch
    hh, ww = image_shape(*ssa.shape, stride)
    img = torch.zeros((hh, ww, IN_CHANNELS), dtype=torch.float32, device=r.device)
    rho = torch.zeros((), dtype=torch.float64, device=r.device)
    rr = r.contiguous()
    ssa._check(ssa.lib.pism_gpu_ssa_learned_pc_input(ssa._h, stride, _ptr(rr), _ptr(img), hh, ww, _ptr(rho)),
               "learned_pc_input")
    return img, rho


def pc_config(c: SSAConfig) -> SSAConfig:
    """the FP64 FGMRES(30) + multigrid set-up the correction works inside"""
    return c.copy(pc_type="mg", precision="fp64", ksp_type="gmres", gmres_restart=30, graphs=2)


def generate_pc(seeds, M: int = 401, samples: int = 4, picard_rtol: float = 1e-2, device: int = 0, log=None):
    """Training pairs of the correction from seeded sheets: each sheet is solved to a Picard
    tolerance of picard_rtol (an iterate on the way to the solution, where the operator has
    the structure the linear solves see), then for `samples` random vectors v the residual
    the multigrid cycle leaves, r = v - A M^-1 v, and the error that removes it, e = A^-1 r
    (a linear solve to 1e-10).  Input: the network image of r (features + the block means
    of D^-1 r / rho); target: e / rho at the cells.  Returns [(x, t, w)] on the device."""
    import torch
    from .ssa import SSAFD
    dev = torch.device("cuda", device)
    out = []
    rng = torch.Generator(device=dev)
    s = None
    try:
        for q, seed in enumerate(seeds):
            g, c, f, _ = training_case(seed, M)
            cfg = pc_config(c).copy(ssafd_relative_convergence=picard_rtol, ksp_rtol=1e-8)
            if s is None:
                s = SSAFD(g, cfg, device=device)
            else:
                s.set_config(cfg)
            s.set_inputs(**{k: f[k] for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")})
            s.set_initial_guess(torch.zeros((M, M, 2), dtype=torch.float64, device=dev))
            s.solve(out=torch.empty((M, M, 2), dtype=torch.float64, device=dev))
            s.set_config(cfg.copy(ksp_rtol=1e-10))
            hh, ww = image_shape(M, M, 1)
            mask = torch.tensor(f["mask"], device=dev)
            w = torch.zeros((hh, ww), dtype=torch.float32, device=dev)
            w[:M, :M] = torch.where((mask == 2) | (mask == 3), 1.0, 0.2).float()
            rng.manual_seed(int(seed))
            for _ in range(samples):
                v = torch.randn((M, M, 2), dtype=torch.float64, device=dev, generator=rng)
                z = torch.empty_like(v)
                s.apply_preconditioner(v, z)
                az = torch.empty_like(v)
                s.apply(z, az)
                r = v - az
                img, rho = pc_input(s, r, 1)
                e = torch.zeros_like(r)
                s.linear_solve_rhs(r, e)
                t = torch.zeros((hh, ww, 2), dtype=torch.float32, device=dev)
                t[:M, :M] = (e / rho).float()
                out.append((img, t, w))
            if log:
                log(f"pc case {q} seed {seed}: {samples} samples")
    finally:
        if s is not None:
            s.close()
    return out
