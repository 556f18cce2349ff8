"""Benchmark: one SSAFD solve on the seeded synthetic 801 x 801 ice sheet (5 km grid).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--size M]

A step is one complete SSA solve (SSAFD::solve: driving stress, hardness, the
Picard loop with its linear solves) of the seeded synthetic sheet (plastic till).
Two solver set-ups run on the same inputs and the same Picard tolerance:

* ``plain``: FP64 throughout, every Picard linear solve to KSP rtol 1e-8
  (BiCGStab + aggregation multigrid), from a zero initial guess;
* ``fast`` (the headline): inexact Picard (early linear solves only as accurate as
  the nonlinear iteration needs, the accepted one to relative residual 1e-6), FP32
  inner BiCGStab + FP32 multigrid inside FP64 iterative refinement, and the learned
  warm start when trained weights are present.

The Picard tolerance defaults to a relative nu*H change of 1e-6, where the fast
answer is within 1e-5 of the converged FP64 solve (``velocity_error_vs_fp64_oracle``
in the line); the configuration text's 1e-4 is timed beside it
(``comparison.accuracy.picard_rtol_1e-4``).  The metric is milliseconds per solve
(lower is better) of ``--mode`` (default fast); the other set-up is timed beside it.
With N GPUs every rank solves its own replica (no data-path collective: the solve
does not shard) and ``value`` is the job's time per solve = max-over-ranks step
time / N.

``--impl reference`` times the native CPU restatement of the reference's path
(oracle/ssafd_cpu.cc + oracle/ksp_cpu.cc: nu*H, drag and the 18-column assembly, then
PETSc's default GMRES(30) / block-Jacobi ILU(0) with one block per host thread) on a
bounded sample of the same solve, the first Picard iterations, scaled to the whole
solve by one complete run of the same restatement on this sheet.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(REPO, "pismv0.7.3_b200")
METRIC = "SSA solve ms at 801² to rel resid 1e-6: learned+FP32 vs plain FP64, 1 B200"
# The headline Picard tolerance: at nu*H change 1e-6 the fast set-up's answer is within 1e-5
# (relative L2 and Linf) of the converged FP64 solve, the accuracy the metric is stated at;
# the configuration text's 1e-4 leaves both set-ups ~1e-3 from it and is reported beside.
HEADLINE_PICARD_RTOL = 1e-6
# fast set-up: lagged multigrid coarse levels (rebuilt once the summed relative nu*H change
# since the last build reaches this).  Off: on the B200 the 801^2 fast solve at Picard 1e-6
# took 655 Krylov iterations / 236 ms rebuilding every iteration, 978 / 265 ms at 0.01 and
# 2261 / 533 ms at 0.05 (its linear solves are 2-3 iterations long, so a weaker coarse
# correction costs more than the rebuild it saves)
FAST_MG_LAG = 0.0
# launch mode of the timed solves (3: the whole Picard loop as one graph, 2: graph-resident
# Krylov loops, bit for bit the same answers; on the B200 the 801^2 fast solve at Picard
# tolerance 1e-6 took 224 ms with 3 and 236 ms with 2); the other one is timed beside it
DEFAULT_GRAPHS = 3
# In-solve DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum, --cache-control
# none) of one inner iteration's kernels on the 801^2 sheet, per (grid, precision, FP32 apply
# kernel) (profiles/inner_iteration_traffic_801.md: the per-launch averages of the kernels)
INNER_ITERATION_TRAFFIC = {(801, "mixed", 2): 96.5e6}


def _package():
    if "pism_b200" in sys.modules:
        return sys.modules["pism_b200"]
    spec = importlib.util.spec_from_file_location("pism_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pism_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return p.get("hbm_gbs", 6650.0), "measured"
    except OSError:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if "Active" in s[2 + k]
                          and not s[2 + k].startswith("Not")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_case(M, pc="mg"):
    _package()
    from pism_b200 import synthetic as S
    dx = 4000e3 / (M - 1)
    g, c, f, meta = S.build_synthetic(M, dx, seed=0)
    c.ksp_rtol = 1e-8
    c.ssafd_relative_convergence = 1e-4
    c.pc_type = pc
    return g, c, f, meta


def fast_config(c, precision="mixed", factor=1.0, rtol_max=1e-1, mg_lag=0.0):
    """The fast set-up: inexact Picard with FP32 inner solves (the linear solve of a Picard
    iteration only as accurate as the last relative nu*H change, at most 1e-1), multigrid
    coarse levels rebuilt once the summed relative nu*H change reaches mg_lag (0: every
    Picard iteration); the accepted linear solve reaches relative residual 1e-6 in FP64."""
    return c.copy(precision=precision, ksp_rtol=1e-6, ksp_rtol_adaptive=True, ksp_rtol_factor=factor,
                  ksp_rtol_max=rtol_max, mg_rebuild_rtol=mg_lag)


def ms_per_step_local(total_ms, steps):
    return total_ms / max(1, steps)


def max_over_ranks(x: float, device=None) -> float:
    """The largest value of x over the ranks of the process group (x itself without one).
    Replicas are timed separately; the job takes as long as its slowest rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_time_per_solve(step_ms_max: float, world: int) -> float:
    """value of the replica run: every rank solves its own sheet in step_ms_max (the
    slowest rank), so the job delivers world solves in that time"""
    return step_ms_max / world


def mg_levels(M):
    """cells of the multigrid levels below the fine grid (2 x 2 aggregation down to <= 4 x 4)"""
    out, mx, my = [], M, M
    while mx > 4 or my > 4:
        mx, my = (mx + 1) // 2 if mx > 4 else mx, (my + 1) // 2 if my > 4 else my
        out.append(mx * my)
    return out


def iteration_bytes(M, precision, apply_kernel=2):
    """Algorithmic HBM bytes of one inner BiCGStab iteration with two V(1,1) cycles: every
    array a kernel reads or writes, once per kernel (halo neighbours counted once), per fine
    cell.  FP32 Krylov (mixed), s = r - alpha v formed where it is read:
      p update: r, v, p read, p written                                      32
      x update: phat, shat, v, t, rhat read; d, r read and written           72
      V-cycle on p, fine restrict: p, D^-1, nu*H, beta, flags                40
      V-cycle on s, fine restrict: r, v, D^-1, nu*H, beta, flags             48
      apply_kernel 2 (fine post-smoothing fused with the apply):
        on p: p, D^-1, nu*H, beta, flags read, phat written; rhat read, v written   64
        on s: r, v, D^-1, nu*H, beta, flags read, shat written; t written           64
      apply_kernel 0 / 1 (separate kernels):
        posts 48 (on p) and 56 (on s); applies: phat, nu*H, beta, flags, rhat read,
        v written 40; shat, nu*H, beta, flags, r, v read, t written 48
    FP64 Krylov: 392 B per cell in the Krylov kernels and 112 per V-cycle on the fine level.
    Every V-cycle adds the first coarse vector written and read (16 B per level-1 cell) and,
    per coarse cell, the nine 2 x 2 blocks, D^-1 and b read by both passes and x written
    (344 B)."""
    N0 = M * M
    lev = mg_levels(M)
    coarse = 2 * (16 * lev[0] + 344 * sum(lev))
    if precision != "mixed":
        return 392 * N0 + 2 * 112 * N0 + coarse
    fine = 32 + 72 + 40 + 48 + (64 + 64 if apply_kernel == 2 else 48 + 56 + 40 + 48)
    return fine * N0 + coarse


def iteration_roofline(s, c, M, stream, flush, dev):
    """one inner Krylov iteration of the solver `s` (inputs set, nu*H at the last solve's):
    a tight linear solve from zero after one untimed one, L2 flushed before it; its
    algorithmic bytes per iteration over the time per iteration"""
    import torch
    s.set_config(c.copy(ksp_rtol=1e-10, ksp_rtol_adaptive=False))
    xk = torch.zeros((M, M, 2), dtype=torch.float64, device=dev)
    s.linear_solve(xk)                     # warm-up
    xk.zero_()
    flush.fill_(1.0)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    lin_its, lin_res = s.linear_solve(xk)
    ev[1].record(stream)
    torch.cuda.synchronize()
    lin_ms = ev[0].elapsed_time(ev[1])
    it_ms = lin_ms / max(1, lin_its)
    it_bytes = iteration_bytes(M, c.precision, c.mixed_apply_kernel)
    return {"achieved": it_bytes / (it_ms * 1e-3) / 1e9, "unit": "GB/s", "bytes_per_launch": it_bytes,
            "launch_ms": it_ms, "timed": f"linear solve to rtol 1e-10: {lin_its} iterations in {lin_ms:.2f} ms"}


def working_set_bytes(M, precision):
    """bytes the inner iteration touches (every array once): the fine level's Krylov vectors,
    nu*H, beta, flags, D^-1 and the multigrid hierarchy"""
    N0, lev = M * M, mg_levels(M)
    krylov = (9 if precision == "mixed" else 9 * 2) * 8 * N0   # r, rhat, p, v, s, t, phat, shat, x
    fine = (8 + 4 + 4 + 16 + 8) * N0                           # FP32 nu*H, beta, flags, D^-1, rhs
    return krylov + fine + (9 * 16 + 16 + 8 + 8) * sum(lev)


def large_roofline(c, stream, flush, dev, peak, M=1601):
    """the inner iteration on a 1601^2 sheet of the same construction (2.5 km): its working
    set is several times the 126 MB L2, so the iteration reads HBM"""
    import torch
    from pism_b200.ssa import SSAFD
    g, cl, f, _ = build_case(M)
    cfg = c.copy(ssafd_relative_convergence=cl.ssafd_relative_convergence)
    s = SSAFD(g, cfg.copy(ssafd_relative_convergence=1e-2, max_iterations_ssafd=300), device=dev.index)
    try:
        s.set_stream(stream.cuda_stream)
        s.set_inputs(**{k: torch.tensor(f[k], dtype=torch.float64, device=dev)
                        for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")})
        s.set_initial_guess(torch.zeros((M, M, 2), dtype=torch.float64, device=dev))
        s.solve(out=torch.empty((M, M, 2), dtype=torch.float64, device=dev))   # nu*H of a partly converged state
        r = iteration_roofline(s, cfg, M, stream, flush, dev)
    finally:
        s.close()
    r.update(grid=[M, M], frac=r["achieved"] / peak, working_set_bytes=working_set_bytes(M, c.precision),
             l2_bytes=torch.cuda.get_device_properties(dev).L2_cache_size)
    return r


def column_roofline(vel, stream, flush, dev, peak, M=801, Mz=41, reps=20):
    """StressBalance::update's 3-D fields (pism_gpu_ssa_stress_balance_3d: ConstantInColumn's
    u and v, the vertical velocity, the volumetric strain heating) on the benchmark sheet with
    Mz levels through 4000 m, from the solved velocity, device outputs.  Algorithmic bytes per
    call: the four [M, M, Mz] FP64 outputs written once plus the velocity, mask, thickness and
    basal melt rate read once (the flow law is isothermal: no enthalpy is read)."""
    import torch
    from pism_b200.config import GridDesc
    from pism_b200.ssa import SSAFD
    g0, cl, f, _ = build_case(M)
    g = GridDesc(g0.Mx, g0.My, g0.Lx, g0.Ly, periodicity=0, z=np.linspace(0.0, 4000.0, Mz))
    s = SSAFD(g, cl, device=dev.index)
    try:
        s.set_stream(stream.cuda_stream)
        s.set_inputs(**{k: torch.tensor(f[k], dtype=torch.float64, device=dev)
                        for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")})
        s.set_initial_guess(vel)
        bmr = torch.full((M, M), 1e-9, dtype=torch.float64, device=dev)
        out = {k: torch.empty((M, M, Mz), dtype=torch.float64, device=dev)
               for k in ("u", "v", "w", "strain_heating")}
        s.stress_balance_3d(bmr, out=out)
        ts = []
        for _ in range(reps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.stress_balance_3d(bmr, out=out)
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
    finally:
        s.close()
    ms = float(np.median(ts))
    nbytes = 4 * 8 * M * M * Mz + M * M * (16 + 1 + 8 + 8)
    achieved = nbytes / (ms * 1e-3) / 1e9
    return {"grid": [M, M, Mz], "ms": ms, "bytes_per_call": nbytes, "achieved": achieved, "unit": "GB/s",
            "peak": peak, "frac": achieved / peak, "bound": "hbm",
            "kernel": "k_stress_balance_3d (one thread per column, results staged per warp in shared memory and "
                      "written coalesced; the call's time includes its argument checks and one stream "
                      "synchronisation)"}


def mass_roofline(vel, stream, flush, dev, peak, M=801, reps=20):
    """The explicit mass-continuity step (pism_gpu_ssa_mass_continuity_step) on the benchmark
    sheet from the solved velocity, one model year, device buffers.  Algorithmic bytes per
    call and cell: velocity 16, mask 1, thickness 8, bed 8, climatic mass balance 8, basal
    melt rate 8, cell area 8 read; thickness, mask, surface and flux divergence 8 each
    written (97 B)."""
    import torch
    from pism_b200.ssa import SSAFD
    g, cl, f, _ = build_case(M)
    s = SSAFD(g, cl, device=dev.index)
    try:
        s.set_stream(stream.cuda_stream)
        s.set_inputs(**{k: torch.tensor(f[k], dtype=torch.float64, device=dev)
                        for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")})
        s.set_initial_guess(vel)
        cmb = torch.full((M, M), 1e-5, dtype=torch.float64, device=dev)
        bmr = torch.full((M, M), 1e-9, dtype=torch.float64, device=dev)
        area = torch.full((M, M), g.dx * g.dy, dtype=torch.float64, device=dev)
        s.mass_continuity_step(3.15e7, cmb, bmr, area)
        ts = []
        for _ in range(reps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.mass_continuity_step(3.15e7, cmb, bmr, area)
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
    finally:
        s.close()
    ms = float(np.median(ts))
    nbytes = 97 * M * M
    achieved = nbytes / (ms * 1e-3) / 1e9
    return {"grid": [M, M], "ms": ms, "bytes_per_call": nbytes, "achieved": achieved, "unit": "GB/s", "peak": peak,
            "frac": achieved / peak, "bound": "hbm",
            "kernel": "k_mass_continuity (one thread per cell, the eight flux totals reduced in the same launch; "
                      "the call's time includes the read-back of the totals and one stream synchronisation)"}


def calving_point(vel, stream, flush, dev, peak, M=801, reps=20):
    """The calving front's consumers of the velocity on the benchmark sheet, device buffers:
    pism_gpu_ssa_strain_rates (principal strain rates and 2-D stresses; algorithmic bytes per
    cell: velocity 16 and mask 1 read, 16 + 24 written, 57 B) and one eigen-calving step
    (pism_gpu_ssa_eigen_calving with K = 1e17 m s over a year, remove_narrow_tongues
    included; its time counts every sweep and the flag read-back after each)."""
    import torch
    from pism_b200.ssa import SSAFD
    g, cl, f, _ = build_case(M)
    s = SSAFD(g, cl, device=dev.index)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)   # noqa: E731
    try:
        s.set_stream(stream.cuda_stream)
        s.set_inputs(**{k: t(f[k]) for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")})
        s.set_initial_guess(vel)
        mask, H = t(f["mask"]), t(f["thickness"])
        href = torch.zeros_like(H)

        def timed(fn):
            fn()
            ts = []
            for _ in range(reps):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            return float(np.median(ts))

        ms_sr = timed(lambda: s.strain_rates(mask, device=True))
        ms_ec = timed(lambda: s.eigen_calving(3.15e7, 1e17, mask, href, H))
        cut = s.eigen_calving(3.15e7, 1e17, mask, href, H)
        changed = int((cut["mask"] != mask).sum().item())
    finally:
        s.close()
    nbytes = 57 * M * M
    achieved = nbytes / (ms_sr * 1e-3) / 1e9
    return {"grid": [M, M], "strain_rates_ms": ms_sr, "bytes_per_call": nbytes, "achieved": achieved,
            "unit": "GB/s", "peak": peak, "frac": achieved / peak, "bound": "hbm",
            "eigen_calving_ms": ms_ec, "cells_cut": changed,
            "kernel": "k_strain_rates (one thread per cell); eigen-calving: k_ec_front, k_ec_cut, k_ec_tongues "
                      "sweeps to their fixed point, k_ec_finish"}


def ssafem_point(dev, stream, reps=3):
    """SSAFEM (pism_gpu_ssafem_solve) at the reference's solver settings on two verification
    grids larger than its regression tests: test J's periodic shelf at 241^2 (one Newton step,
    a linear problem) and test I's plastic-till stream at 5 x 481 (Newton from zero)."""
    import torch
    from pism_b200 import verification as Ver
    from pism_b200.ssa import SSAFEM
    out = {}
    for name, (g, c, f), exact in (("test_j_241", Ver.build_test_j(241, 241), Ver.exact_velocity_j),
                                   ("test_i_5x481", Ver.build_test_i(My=481), Ver.exact_velocity_i)):
        s = SSAFEM(g, c, device=dev.index)
        try:
            s.set_stream(stream.cuda_stream)
            s.set_inputs(**{k: f[k] for k in ("thickness", "surface", "bed", "mask", "tauc")},
                         bc_mask=f["bc_mask"], bc_values=f["bc_values"])
            ts = []
            for _ in range(reps):
                s.set_initial_guess(np.zeros((g.Mx, g.My, 2)))
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                vel = s.solve()
                ts.append((time.perf_counter() - t0) * 1e3)
            st = s.stats()
        finally:
            s.close()
        err = Ver.report(vel, exact(g))
        out[name] = {"ms": float(np.median(ts)), "newton_iterations": st["newton_iterations"],
                     "cg_iterations": st["ksp_iterations"], "converged": st["converged"],
                     "maxvector_error_m_per_year": err["maxvector"]}
    out["note"] = "wall time of the call (host loop with a read-back per Newton step and CG batch)"
    return out


# The host-core cost of the whole reference solve is sampled: the first CPU_SAMPLE_PICARD
# Picard iterations of the native restatement (oracle/ssafd_cpu.cc: nu*H, drag, 18-column
# assembly, PETSc-style GMRES(30) + block Jacobi / ILU(0), norms) run on the host cores, and
# the whole solve is estimated by a cost model: Picard iteration k costs (c + its_k) units, its_k
# its GMRES iterations and c the per-Picard set-up (ILU(0) factorisation, assembly) in GMRES
# iterations.  The unit is the median over the sampled iterations of t_k / (c + its_k) (one
# iteration slowed by another process does not move it); the whole solve costs
# (n c + sum its_k) units with n and sum its_k from one complete run of the same restatement on
# this sheet (KSP rtol 1e-8 from a zero guess; the tolerance-1e-4 solve is the prefix of the
# tolerance-1e-6 one), c fitted on that run (least squares with 4-MAD outlier rejection).
CPU_FULL_RUN_801 = {
    "threads": 8,
    "picard_iterations": {"1e-06": 359, "0.0001": 184},
    "ksp_iterations": {"1e-06": 27936, "0.0001": 22646},
    "setup_iterations": 13.6,
}
CPU_SAMPLE_PICARD = 3


def cpu_estimate(prepare_s, sample, picard_rtol, full=None):
    """(estimated ms of the whole CPU solve, how) from the set-up seconds and the sampled
    Picard iterations' (seconds, GMRES iterations)"""
    full = full if full is not None else CPU_FULL_RUN_801
    if full is None or not sample:
        return None, "no complete CPU run on record"
    key = f"{picard_rtol:g}"
    if key not in full["ksp_iterations"]:
        return None, f"no complete CPU run at Picard tolerance {key}"
    c = full["setup_iterations"]
    n, its = full["picard_iterations"][key], full["ksp_iterations"][key]
    unit = float(np.median([t / (c + k) for t, k in sample]))
    est = prepare_s + unit * (its + n * c)
    how = (f"first {len(sample)} Picard iterations timed on the host cores "
           f"({sum(t for t, _ in sample):.1f} s, {sum(k for _, k in sample)} GMRES iterations): median cost "
           f"{unit * 1e3:.2f} ms per GMRES iteration with {c:g} iterations of set-up per Picard iteration, "
           f"times the {n} Picard and {its} GMRES iterations of one complete run of the same restatement on "
           f"this sheet at Picard tolerance {key}")
    return est * 1e3, how


def cpu_reference_sample(M, picard_sample, nthreads, picard_rtol):
    """The native CPU restatement of the reference's Picard loop (oracle/ssafd_cpu.cc) on the
    host cores: driving stress / right-hand side / hardness (oracle.prepare), then
    `picard_sample` Picard iterations from a zero guess (nu*H, drag, assembly, PETSc-style
    GMRES(30) + block Jacobi ILU(0) with one block per thread, norms).  Returns (set-up
    seconds, [(seconds, GMRES iterations) per Picard iteration])."""
    sys.path.insert(0, REPO)
    from oracle import ssafd_oracle as O
    g, c, f, _ = build_case(M)
    c.ssafd_relative_convergence = picard_rtol
    G, Cc, I = O.from_case(g, c, f)
    t0 = time.perf_counter()
    o = O.SSAFDOracle(G, Cc, I)
    o.prepare()
    t1 = time.perf_counter()
    _, info = O.picard_native(G, Cc, I, o.hardness, o.b, np.zeros((M, M, 2)), Cc.epsilon_ssa, nranks=nthreads,
                              nthreads=nthreads, ksp_rtol=c.ksp_rtol, max_iterations=picard_sample,
                              picard_rtol=picard_rtol)
    total = time.perf_counter() - t1
    per = [a + b + d for a, b, d in zip(info["t_nuH"], info["t_assemble"], info["t_ksp"])]
    rest = (total - sum(per)) / max(1, len(per))   # norms, tests and the copies around them
    return t1 - t0, [(t + rest, int(k)) for t, k in zip(per, info["ksp_iterations"])]


def cpu_baseline(M, picard_rtol, nthreads, picard_gpu=None):
    """the cpu_baseline object: the host-core sample and its whole-solve estimate"""
    prep, sample = cpu_reference_sample(M, CPU_SAMPLE_PICARD, nthreads, picard_rtol)
    est, how = (cpu_estimate(prep, sample, picard_rtol) if M == 801 else (None, "no complete CPU run at this size"))
    if est is None and picard_gpu and sample:
        dt = sum(t for t, _ in sample)
        est = (prep + dt / len(sample) * picard_gpu) * 1e3
        how = (f"first {len(sample)} Picard iterations timed on the host cores ({dt:.1f} s), scaled by the "
               f"iteration count of the plain GPU solve ({picard_gpu}; {how})")
    return {"value": est, "unit": "ms", "cores": nthreads, "kind": "port", "sample": how}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    vals, sample = [], None
    for k in range(args.warmup + args.steps):
        cb = cpu_baseline(args.size, args.picard_rtol, nthreads, picard_gpu=args.picard_full or None)
        if k >= args.warmup:
            vals.append(cb["value"])
            sample = cb["sample"]
    v = float(np.mean(vals)) if all(x is not None for x in vals) else None
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"SSAFD solve, synthetic ice sheet {args.size}x{args.size} at "
                               f"{4000 / (args.size - 1):.0f} km, plastic till, Picard {args.picard_rtol:g}, KSP 1e-8",
                   "grid": [args.size, args.size], "seed": 0,
                   "implementation": "native restatement of SSAFD's Picard loop with PETSc's default KSP "
                                     "(oracle/ssafd_cpu.cc, oracle/ksp_cpu.cc), one block-Jacobi block per thread"},
        "cpu_baseline": {"value": v, "unit": "ms", "cores": nthreads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def members_of_rank(rank: int, world: int, per_gpu: int) -> list:
    """the ensemble members rank `rank` of `world` solves: a contiguous block of `per_gpu`
    member indices, disjoint between ranks, the whole job covering 0 .. world * per_gpu - 1"""
    if not (0 <= rank < world) or per_gpu < 0:
        raise ValueError("0 <= rank < world and per_gpu >= 0")
    return list(range(rank * per_gpu, (rank + 1) * per_gpu))


def ensemble_member(q, M=401):
    """member q of the ensemble: a seeded 401^2 sheet (10 km) with its own ice temperature
    ~ U[-20, -2] C and tau_c median ~ U[20, 200] kPa (seeds disjoint from the training set)"""
    _package()
    from pism_b200 import synthetic as S
    rng = np.random.Generator(np.random.PCG64(77_000 + q))
    T, med = rng.uniform(-20.0, -2.0), rng.uniform(20e3, 200e3)
    g, c, f, meta = S.build_synthetic(M, 4000e3 / (M - 1), seed=700_000 + q, temperature_c=T, tauc_median=med)
    return g, c, f, {"T": T, "tauc_median": med}


def ensemble_point(stream, flush, dev, members=16, steps=2):
    """members/s of pism_gpu_ssa_solve_batch on `members` seeded 401^2 sheets (the ensemble
    workload's members 0 .. members-1, fast set-up, learned guess), device-timed, L2 flushed
    before each batch: the ensemble configuration in the default bench line"""
    import torch
    from pism_b200 import learned as Lrn
    from pism_b200.ssa import SSAFD
    M = 401
    names = ("thickness", "surface", "bed", "mask", "tauc", "melange")
    cases = [ensemble_member(q, M) for q in range(members)]
    g, c0 = cases[0][0], cases[0][1]
    mem = [{**{k: torch.tensor(f[k], dtype=torch.float64, device=dev) for k in names},
            "ice_softness": c.ice_softness, "velocity": torch.zeros((M, M, 2), dtype=torch.float64, device=dev)}
           for _, c, f, _ in cases]
    hh, ww = Lrn.image_shape(M, M, 1)
    net = Lrn.UNet(1, hh, ww, device=dev.index, params=np.load(Lrn.DEFAULT_WEIGHTS)["params"])
    net.set_stream(stream.cuda_stream)
    s = SSAFD(g, fast_config(c0), device=dev.index)
    try:
        s.set_stream(stream.cuda_stream)
        s.solve_batch(mem[:2], net=net, stride=1)   # warm-up
        ts, stats = [], None
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, stats = s.solve_batch(mem, net=net, stride=1)
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
    finally:
        s.close()
        net.close()
    ms = float(np.mean(ts))
    return {"members": members, "grid": [M, M], "ms_per_batch": ms, "members_per_s": members / (ms * 1e-3),
            "converged": int(sum(st["converged"] for st in stats)),
            "picard_iterations": [st["picard_iterations"] for st in stats],
            "how": "pism_gpu_ssa_solve_batch, members in turn on one handle (bench.py --workload ensemble "
                   "runs the 64-member configuration with its accuracy check)"}


def run_ensemble(args):
    """--workload ensemble: pism_gpu_ssa_solve_batch over the members of this rank (the
    fast set-up with the learned guess), members/s of the whole job; each member's
    velocity error against the plain FP64 solve of the same member."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    _package()
    from pism_b200 import learned as Lrn
    from pism_b200.ssa import SSAFD
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    M = 401
    mine = members_of_rank(rank, world, args.members)   # weak scaling: members per GPU fixed
    names = ("thickness", "surface", "bed", "mask", "tauc", "melange")
    cases = [ensemble_member(q, M) for q in mine]
    g, c0 = cases[0][0], cases[0][1]
    c_fast = fast_config(c0)
    mem = [{**{k: torch.tensor(f[k], dtype=torch.float64, device=dev) for k in names},
            "ice_softness": c.ice_softness, "velocity": torch.zeros((M, M, 2), dtype=torch.float64, device=dev)}
           for _, c, f, _ in cases]
    hh, ww = Lrn.image_shape(M, M, 1)
    net = Lrn.UNet(1, hh, ww, device=local, params=np.load(Lrn.DEFAULT_WEIGHTS)["params"])
    net.set_stream(stream.cuda_stream)
    s = SSAFD(g, c_fast, device=local)
    s.set_stream(stream.cuda_stream)
    s.solve_batch(mem[:2], net=net, stride=1)   # warm-up
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        dist.barrier()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        vels, stats = s.solve_batch(mem, net=net, stride=1)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    step_ms = max_over_ranks(float(np.mean(times)), dev)
    value = len(mine) * world / (step_ms * 1e-3)
    # end to end: host inputs and outputs through the same call
    hmem = [{**{k: f[k] for k in names}, "ice_softness": c.ice_softness, "velocity": np.zeros((M, M, 2))}
            for _, c, f, _ in cases]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.solve_batch(hmem, net=net, stride=1)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, dev)
    # accuracy: the plain FP64 solve of every member
    errs = []
    plain = SSAFD(g, c0, device=local)
    plain.set_stream(stream.cuda_stream)
    for q, (_, c, f, meta) in enumerate(cases):
        plain.set_config(c)
        plain.set_inputs(**{k: mem[q][k] for k in names})
        plain.set_initial_guess(torch.zeros((M, M, 2), dtype=torch.float64, device=dev))
        ref = plain.solve(out=torch.empty((M, M, 2), dtype=torch.float64, device=dev))
        errs.append(float((vels[q] - ref).norm() / ref.norm()))
    plain.close()
    s.close()
    net.close()
    line = {
        "metric": f"ensemble members solved/s ({args.members} x {M}^2 per GPU, learned+FP32)", "value": value,
        "unit": "members/s", "n_gpus": world, "steps": args.steps, "warmup": 1, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": f"ensemble of {args.members} seeded {M}x{M} sheets at 10 km per GPU, temperature "
                               "U[-20,-2] C and tau_c median U[20,200] kPa per member, solved by "
                               "pism_gpu_ssa_solve_batch (fast set-up, learned guess)",
                   "members_per_gpu": args.members, "l2": "flushed (256 MB write) between steps",
                   "parallelism": f"members sharded over {world} GPU(s)"},
        "members": {"picard_iterations": [st["picard_iterations"] for st in stats],
                    "converged": sum(st["converged"] for st in stats),
                    "rel_l2_error_vs_plain_fp64": {"max": max(errs), "median": float(np.median(errs))}},
        "e2e": {"value": len(mine) * world / (e2e_ms * 1e-3), "unit": "members/s",
                "h2d_bytes_per_step": len(mine) * len(names) * M * M * 8,
                "d2h_bytes_per_step": len(mine) * M * M * 16},
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--size", type=int, default=801)
    ap.add_argument("--picard-full", type=int, default=0,
                    help="reference arm away from 801^2: Picard iterations to scale the CPU sample by")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--apply-launches", type=int, default=50)
    ap.add_argument("--pc", default="mg", choices=["mg", "bjacobi"])
    ap.add_argument("--mg-omega", type=float, default=None)
    ap.add_argument("--mg-correction", type=float, default=None)
    ap.add_argument("--verbosity", type=int, default=0)
    ap.add_argument("--mode", default="fast", choices=["fast", "plain"])
    ap.add_argument("--ksp", default=None, choices=["bicgstab", "gmres"], help="override the Krylov method")
    ap.add_argument("--gmres-restart", type=int, default=None)
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="override the mode's precision (fast: mixed, plain: fp64)")
    ap.add_argument("--inner-rtol", type=float, default=None)
    ap.add_argument("--no-learned", action="store_true", help="fast set-up from a zero initial guess")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the converged FP64 reference solve")
    ap.add_argument("--no-compare", action="store_true", help="skip the other set-up (and the accuracy reference)")
    ap.add_argument("--no-large", action="store_true", help="skip the larger-than-L2 roofline point")
    ap.add_argument("--workload", default="solve", choices=["solve", "ensemble"],
                    help="ensemble: members solved/s of a 64-member 401^2 ensemble (its own JSON line)")
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--picard-rtol", type=float, default=HEADLINE_PICARD_RTOL,
                    help="Picard nu*H tolerance of both set-ups (default 1e-6: the tolerance at which the fast "
                         "answer is within 1e-5 of the converged FP64 solve)")
    ap.add_argument("--profile", action="store_true",
                    help="time the solve only (no end-to-end, roofline, comparison or CPU runs): for kernel profilers")
    ap.add_argument("--mg-post-blocks", type=int, default=None, choices=[1, 2, 3, 4],
                    help="resident blocks per SM the coarse-level post-smoothing grid is sized for (default 4)")
    ap.add_argument("--graphs", type=int, default=DEFAULT_GRAPHS, choices=[0, 1, 2, 3],
                    help="Krylov launch mode: 2 graph-resident loops, 1 replayed graphs, 0 direct (for profilers), "
                         "3 the whole Picard loop as one graph")
    ap.add_argument("--ksp-factor", type=float, default=1.0,
                    help="fast set-up: KSP rtol of a Picard iteration = factor x the last relative nu*H change")
    ap.add_argument("--ksp-max", type=float, default=1e-1, help="fast set-up: loosest KSP rtol of a Picard iteration")
    ap.add_argument("--mg-small-kernel", type=int, default=0, choices=[0, 1, 2],
                    help="multigrid small levels: 0 staged from L2 per step, 1 held in the cluster's shared memory, "
                         "2 as 0 from the first level of <= 16384 cells")
    ap.add_argument("--apply-kernel", type=int, default=2, choices=[0, 1, 2],
                    help="mixed precision, the FP32 operator apply after each V-cycle: 0 plain tile loads, "
                         "1 bulk-copy staged tiles, 2 fused into the V-cycle's fine-level pass")
    ap.add_argument("--mg-lag", type=float, default=FAST_MG_LAG,
                    help="fast set-up: rebuild the multigrid coarse levels once the summed relative nu*H change "
                         "reaches this (0: every Picard iteration)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ensemble":
        return run_ensemble(args)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    _package()
    from pism_b200.ssa import SSAFD

    g, c_plain, f, meta = build_case(args.size, args.pc)
    if args.mg_omega is not None:
        c_plain.mg_omega = args.mg_omega
    if args.mg_correction is not None:
        c_plain.mg_correction = args.mg_correction
    c_plain.verbosity = args.verbosity
    c_plain.ssafd_relative_convergence = args.picard_rtol
    c_plain.max_iterations_ssafd = 5000
    c_plain.graphs = args.graphs
    if args.mg_post_blocks is not None:
        c_plain.mg_post_blocks_per_sm = args.mg_post_blocks
    c_plain.mg_small_kernel = args.mg_small_kernel
    c_plain.mixed_apply_kernel = args.apply_kernel
    c_fast = fast_config(c_plain, factor=args.ksp_factor, rtol_max=args.ksp_max, mg_lag=args.mg_lag)
    if args.inner_rtol is not None:
        c_fast.mixed_inner_rtol = args.inner_rtol
    c, c_other = (c_fast, c_plain) if args.mode == "fast" else (c_plain, c_fast)
    if args.precision is not None:
        c.precision = args.precision
    if args.ksp is not None:
        c.ksp_type = args.ksp
        if args.ksp == "gmres":
            c.precision = "fp64"
            c.graphs = min(c.graphs, 2)
    if args.gmres_restart is not None:
        c.gmres_restart = args.gmres_restart
    M = args.size
    N = M * M
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)      # a real stream: the solver and the events share it
    torch.cuda.set_stream(stream)
    names = ("thickness", "surface", "bed", "mask", "tauc", "melange")
    dfields = {k: torch.tensor(f[k], dtype=torch.float64, device=dev) for k in names}
    zero = torch.zeros((M, M, 2), dtype=torch.float64, device=dev)
    out = torch.empty((M, M, 2), dtype=torch.float64, device=dev)
    s = SSAFD(g, c, device=local)
    s.set_stream(stream.cuda_stream)
    s.set_inputs(**dfields)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)   # > L2 (126 MB)

    # the learned warm start (fast set-up): features at stride 2 above 600^2 cells a side
    from pism_b200 import learned as Lrn
    net = None
    stride = 2 if M >= 600 else 1
    if args.mode == "fast" and not args.no_learned and os.path.exists(Lrn.DEFAULT_WEIGHTS):
        hh, ww = Lrn.image_shape(M, M, stride)
        net = Lrn.UNet(1, hh, ww, device=local, params=np.load(Lrn.DEFAULT_WEIGHTS)["params"])
        net.set_stream(stream.cuda_stream)

    def prime(solver, learned, host_zero=None):
        """the initial guess of one solve: the network's prediction, or zero"""
        if learned:
            Lrn.learned_guess(solver, net, stride)
        else:
            solver.set_initial_guess(zero if host_zero is None else host_zero)

    def step():
        prime(s, net is not None)
        s.solve(out=out)

    def timed(solver, learned, result, reps=2):
        """mean device time of `reps` solves after one untimed one, L2 flushed before each"""
        prime(solver, learned)
        solver.solve(out=result)
        ts = []
        for _ in range(reps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            prime(solver, learned)
            solver.solve(out=result)
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.mean(ts)), solver.stats()

    for _ in range(args.warmup):
        step()
    st = s.stats()

    # end to end through the C-ABI with pinned host buffers, every step: H2D inputs, the
    # initial guess, the solve, D2H velocity. One such solve follows each device-timed solve,
    # so both see the same clocks, host load and cache state.
    hfields = {k: torch.tensor(f[k], dtype=torch.float64).pin_memory() for k in names}
    hzero = torch.zeros((M, M, 2), dtype=torch.float64).pin_memory()
    hout = torch.empty((M, M, 2), dtype=torch.float64).pin_memory()
    h2d = sum(v.numel() * 8 for v in hfields.values()) + (0 if net is not None else hzero.numel() * 8)
    d2h = hout.numel() * 8
    e2e_ms, e2e_steps = 0.0, []

    def e2e_step():
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.set_inputs(**{k: v.numpy() for k, v in hfields.items()})
        prime(s, net is not None, hzero.numpy())
        s.solve(out=hout.numpy())
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3

    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    launches = 0
    picard, ksp, refine, rebuilds, step_ms = [], [], [], [], []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        step_ms.append(e0.elapsed_time(e1))
        st = s.stats()
        # the solver's own count, plus the learned guess: features, 18 network kernels, velocity
        launches += st["kernel_launches"] + (20 if net is not None else 0)
        picard.append(st["picard_iterations"])
        ksp.append(st["ksp_iterations"])
        refine.append(st["refinement_steps"])
        rebuilds.append(st["mg_rebuilds"])
        if not args.profile:
            e2e_steps.append(e2e_step())
            e2e_ms += e2e_steps[-1]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    vel_mode = out.clone()
    if args.profile:
        sampler.stop()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": ms_per_step_local(total_ms, args.steps), "unit": "ms",
                              "profile": True, "solver": {"picard_iterations": picard, "ksp_iterations": ksp}}))
        s.close()
        return 0

    ms_per_step = max_over_ranks(total_ms, dev) / args.steps
    value = job_time_per_solve(ms_per_step, world)

    def errors(a, ref):
        d = a - ref
        return {"l2_rel": float(d.norm() / ref.norm()), "linf_rel": float(d.abs().max() / ref.abs().max())}

    other_ms, st_other, vel_error, accuracy, headline_error = None, {"picard_iterations": None,
                                                                     "ksp_iterations": None}, None, None, None
    if not args.no_compare:
        # the other set-up on the same inputs and tolerance, timed like a step
        s_other = SSAFD(g, c_other, device=local)
        s_other.set_stream(stream.cuda_stream)
        s_other.set_inputs(**dfields)
        out_other = torch.empty_like(out)
        other_ms, st_other = timed(s_other, args.mode == "plain" and net is not None, out_other)
        s_other.close()
        vel_fast, vel_plain = (vel_mode, out_other) if args.mode == "fast" else (out_other, vel_mode)
        vel_error = errors(vel_fast, vel_plain)
        if not args.no_accuracy:
            # the FP64 oracle answer: an FP64 Picard iteration continued from the plain answer to
            # a nu*H change 100 x below the set-ups' tolerance (the GPU FP64 path equals the CPU
            # oracle to 1e-8 relative, tests/test_gpu_parity*.py)
            c_conv = c_plain.copy(ssafd_relative_convergence=min(1e-8, 0.01 * args.picard_rtol), ksp_rtol=1e-10,
                                  ksp_rtol_adaptive=True, ksp_rtol_factor=0.1, ksp_rtol_max=1e-2,
                                  max_iterations_ssafd=20000, precision="fp64", graphs=2)
            s_ref = SSAFD(g, c_conv, device=local)
            s_ref.set_stream(stream.cuda_stream)
            s_ref.set_inputs(**dfields)
            s_ref.set_initial_guess(vel_plain)
            vel_conv = torch.empty_like(out)
            s_ref.solve(out=vel_conv)
            st_ref = s_ref.stats()
            s_ref.close()
            accuracy = {"reference": f"FP64 Picard continued from the plain answer to nu*H change "
                                     f"{c_conv.ssafd_relative_convergence:g}, KSP rtol 1e-10",
                        "reference_picard_iterations": st_ref["picard_iterations"],
                        "reference_converged": st_ref["converged"],
                        "plain_vs_reference": errors(vel_plain, vel_conv),
                        "fast_vs_reference": errors(vel_fast, vel_conv)}
            headline_error = accuracy["fast_vs_reference" if args.mode == "fast" else "plain_vs_reference"]
            # both set-ups at the configuration text's Picard tolerance 1e-4, against the same answer
            if args.picard_rtol != 1e-4:
                o4 = torch.empty_like(out)
                pair = {}
                for nm, cfg, learned in (("fast", c_fast, net is not None), ("plain", c_plain, False)):
                    h = SSAFD(g, cfg.copy(ssafd_relative_convergence=1e-4, max_iterations_ssafd=300), device=local)
                    h.set_stream(stream.cuda_stream)
                    h.set_inputs(**dfields)
                    t, sh = timed(h, learned, o4)
                    h.close()
                    pair[nm + "_ms"] = t
                    pair[nm + "_picard_iterations"] = sh["picard_iterations"]
                    pair[nm + "_vs_reference"] = errors(o4, vel_conv)
                pair["plain_over_fast"] = pair["plain_ms"] / pair["fast_ms"]
                accuracy["picard_rtol_1e-4"] = pair

    if not e2e_steps:                     # --steps 0: one end-to-end solve all the same
        e2e_steps.append(e2e_step())
        e2e_ms += e2e_steps[-1]
    e2e_ms /= len(e2e_steps)
    clocks = sampler.stop()   # sampled over the timed steps and the end-to-end steps alike
    e2e_value = job_time_per_solve(max_over_ranks(e2e_ms, dev), world)
    e2e_same = bool(torch.equal(hout, vel_mode.cpu()))

    # Roofline of the hot loop: one inner BiCGStab + multigrid iteration (the kernels that
    # repeat ~1000 times per fast solve), timed live on a tight linear solve at the final nu*H
    peak, peak_kind = _peaks()
    roof = iteration_roofline(s, c, M, stream, flush, dev)
    s.set_config(c)
    roof.update(peak=peak, frac=roof["achieved"] / peak, peak_kind=peak_kind, bound="hbm",
                traffic=INNER_ITERATION_TRAFFIC.get((M, c.precision, c.mixed_apply_kernel)))
    roof["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the iteration's kernels, "
                              "in-solve (--cache-control none), profiles/inner_iteration_traffic_801.md"
                              if roof["traffic"] is not None else None)
    fine_last = {2: "k_mg0_post_apply (the post-smoothing fused with the FP32 apply)",
                 1: "k_mg0_post, then k32_apply with bulk-copy-staged tiles",
                 0: "k_mg0_post, then k32_apply"}[c.mixed_apply_kernel]
    roof["kernel"] = (f"one inner BiCGStab + V(1,1) multigrid iteration: k32_p, k32_x + 2 x (k_mg0_restrict, "
                      f"k_mgc_restrict x3, k_mg_small_cycle, k_mgc_post x3, {fine_last})"
                      if c.precision == "mixed" else "one BiCGStab + V(1,1) multigrid iteration (FP64 Krylov vectors)")
    # the FP64 matrix-free apply alone, each launch timed with L2 flushed before it (HBM-bound)
    x = torch.randn((M, M, 2), dtype=torch.float64, device=dev) * 1e-5
    y = torch.empty_like(x)
    for _ in range(5):
        s.apply(x, y)
    apply_ms = []
    for _ in range(args.apply_launches):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.apply(x, y)
        e1.record(stream)
        torch.cuda.synchronize()
        apply_ms.append(e0.elapsed_time(e1))
    apply_ms = float(np.median(apply_ms))
    apply_bytes = 60 * N   # x 16, nu*H 16, beta 8, flags 4, y 16 per cell (neighbours counted once)
    roof["fp64_apply"] = {"achieved": apply_bytes / (apply_ms * 1e-3) / 1e9, "bytes_per_launch": apply_bytes,
                          "launch_ms": apply_ms, "frac": apply_bytes / (apply_ms * 1e-3) / 1e9 / peak,
                          "cache": "cold: L2 flushed (256 MB write) before each launch, median of launches"}

    line = {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if c.precision == "fp64" else "f64+f32", "data": "synthetic",
        "config": {"workload": f"SSAFD solve, synthetic ice sheet {M}x{M} at {4000 / (M - 1):.0f} km, plastic till, "
                               f"Picard {c.ssafd_relative_convergence:g}; {args.mode} set-up",
                   "mode": args.mode, "grid": [M, M], "seed": 0, "precision": c.precision,
                   "ksp": f"{'FGMRES(%d)' % c.gmres_restart if c.ksp_type == 'gmres' else 'BiCGStab'} + "
                          f"{'aggregation multigrid' if args.pc == 'mg' else 'block Jacobi'}",
                   "ksp_rtol": c.ksp_rtol, "ksp_rtol_adaptive": bool(c.ksp_rtol_adaptive),
                   "picard_rtol": c.ssafd_relative_convergence, "graphs": c.graphs,
                   "mg_rebuild_rtol": c.mg_rebuild_rtol, "mg_small_kernel": c.mg_small_kernel,
                   "mixed_apply_kernel": c.mixed_apply_kernel,
                   "warm_start": (f"learned (U-Net, features at stride {stride})" if net is not None else "zero"),
                   "l2": "flushed (256 MB write) between steps",
                   "parallelism": f"replicas x{world}"},
        "velocity_error_vs_fp64_oracle": headline_error,
        "solver": {"picard_iterations": picard, "ksp_iterations": ksp, "converged": st["converged"],
                   "refinement_steps": refine, "mg_rebuilds": rebuilds, "step_ms": step_ms,
                   "strategy": st["strategy"], "final_linear_residual": st["final_linear_residual"]},
        "comparison": {"other_mode": "plain" if args.mode == "fast" else "fast", "other_ms": other_ms,
                       "other_picard_iterations": st_other["picard_iterations"],
                       "other_ksp_iterations": st_other["ksp_iterations"],
                       "plain_over_fast": (None if other_ms is None else
                                           (other_ms / ms_per_step) if args.mode == "fast" else (ms_per_step / other_ms)),
                       "fast_velocity_error_vs_plain_fp64": vel_error,
                       "accuracy": accuracy},
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": max(1, args.steps), "step_ms": e2e_steps, "same_velocity_as_timed": e2e_same},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    # the same solve in the other launch mode (graph-resident loops <-> the whole Picard loop
    # as one CUDA graph), after all of the above: timed like a step and checked bit for bit
    # against the timed answer; an error is reported, not raised
    if not args.no_compare and c.graphs in (2, 3) and c.ksp_type == "bicgstab":
        other_graphs = 5 - c.graphs
        try:
            s.set_config(c.copy(graphs=other_graphs))
            o3 = torch.empty_like(out)
            t3, st3 = timed(s, net is not None, o3)
            line["comparison"]["launch_mode"] = {
                "graphs": other_graphs, "ms": t3, "timed_mode_ms": ms_per_step_local(total_ms, args.steps),
                "bitwise_equal": bool(torch.equal(o3, vel_mode)), "picard_iterations": st3["picard_iterations"],
                "kernel_launches": st3["kernel_launches"]}
        except Exception as e:   # noqa: BLE001 - reported in the line
            line["comparison"]["launch_mode"] = {"graphs": other_graphs, "error": str(e)[:200]}
        finally:
            try:
                s.set_config(c)
            except Exception:   # noqa: BLE001
                pass
    # the larger-than-L2 roofline point: the same iteration on a 1601^2 sheet (working set
    # ~4x the 801^2 one, well above the 126 MB L2)
    if not args.no_large and M == 801:
        try:
            line["roofline"]["large"] = large_roofline(c, stream, flush, dev, peak)
        except Exception as e:   # noqa: BLE001 - reported in the line
            line["roofline"]["large"] = {"error": str(e)[:200]}
    # the stress balance's 3-D fields from the timed solve's velocity
    if not args.no_large and M == 801:
        try:
            line["stress_balance_3d"] = column_roofline(vel_mode, stream, flush, dev, peak)
        except Exception as e:   # noqa: BLE001 - reported in the line
            line["stress_balance_3d"] = {"error": str(e)[:200]}
        try:
            line["mass_continuity"] = mass_roofline(vel_mode, stream, flush, dev, peak)
        except Exception as e:   # noqa: BLE001 - reported in the line
            line["mass_continuity"] = {"error": str(e)[:200]}
        try:
            line["calving_front"] = calving_point(vel_mode, stream, flush, dev, peak)
        except Exception as e:   # noqa: BLE001 - reported in the line
            line["calving_front"] = {"error": str(e)[:200]}
        try:
            line["ssafem"] = ssafem_point(dev, stream)
        except Exception as e:   # noqa: BLE001 - reported in the line
            line["ssafem"] = {"error": str(e)[:200]}
        try:
            line["ensemble"] = ensemble_point(stream, flush, dev)
        except Exception as e:   # noqa: BLE001 - reported in the line
            line["ensemble"] = {"error": str(e)[:200]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        plain_picard = st_other["picard_iterations"] if args.mode == "fast" else picard[-1]
        line["cpu_baseline"] = cpu_baseline(M, c.ssafd_relative_convergence, nthreads, picard_gpu=plain_picard)
    if rank == 0:
        print(json.dumps(line))
    mode_error = "error" in line["comparison"].get("launch_mode", {})
    try:
        s.close()
        if net is not None:
            net.close()
    except Exception:   # noqa: BLE001 - after a reported launch-mode error the line stands
        if not mode_error:
            raise
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
