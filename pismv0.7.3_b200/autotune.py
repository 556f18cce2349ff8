"""The project's autotuner: choose the fastest launch configuration of a workload by timing
the candidates on the device, check that each candidate gives the answer of the first
(default) one, and remember the choice per (device, library build, workload).

    tuner = Autotuner("tuning.json")
    best = tuner.choose({"workload": "ssa solve", "config": cfg_dict},
                        [{"graphs": 2}, {"graphs": 3}],
                        run=lambda cand: solve_with(cand),          # returns the answer
                        verify=lambda cand, out, ref: torch.equal(out, ref))

Each candidate runs `warmup` untimed times, then `repeats` timed times; its time is the
median.  Timing is done with CUDA events on the current stream around the call, with a
synchronize on both sides (the solver calls return with their work complete).  The first
candidate is the reference: with a `verify` callback, every other candidate's last answer is
compared with the reference's and a candidate that fails is never chosen.  Ties go to the
earlier candidate, so list the default first.  The cache is a JSON file keyed by the device
name, a fingerprint of the solver library and the workload description (which should hold
the whole solver configuration); a cached choice is returned without running anything, as
long as it is still one of the candidates.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os
import statistics
from typing import Any, Callable, Optional


def cuda_event_timer(run: Callable[[], Any]) -> float:
    """Milliseconds of one call, CUDA events on the current stream."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run()
    e1.record()
    torch.cuda.synchronize()
    return float(e0.elapsed_time(e1))


def device_name() -> str:
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def library_fingerprint(path: Optional[str] = None) -> str:
    """sha256 (first 16 hex digits) of the solver library's file: a choice made with another
    build of the kernels is not reused"""
    if path is None:
        from . import _capi
        path = _capi.LIB_PATH
    h = hashlib.sha256()
    try:
        with open(path, "rb") as fh:
            for block in iter(lambda: fh.read(1 << 20), b""):
                h.update(block)
    except OSError:
        return "missing"
    return h.hexdigest()[:16]


def config_key(config) -> dict:
    """the whole solver configuration as a JSON-able dict (dataclass fields)"""
    return {k: v for k, v in dataclasses.asdict(config).items()}


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, repeats: int = 3, warmup: int = 1,
                 timer: Callable[[Callable[[], Any]], float] = cuda_event_timer,
                 device: Optional[Callable[[], str]] = None, library: Optional[Callable[[], str]] = None):
        if repeats < 1 or warmup < 0:
            raise ValueError("repeats >= 1 and warmup >= 0")
        self.cache_path = cache_path
        self.repeats = repeats
        self.warmup = warmup
        self.timer = timer
        self.device = device or device_name
        self.library = library or library_fingerprint
        self.last_times: dict[str, float] = {}
        self.last_rejected: list[dict] = []
        self._cache = self._load()

    def _load(self) -> dict:
        if self.cache_path and os.path.exists(self.cache_path):
            with open(self.cache_path) as fh:
                return json.load(fh)
        return {}

    def _save(self):
        if not self.cache_path:
            return
        d = os.path.dirname(os.path.abspath(self.cache_path))
        os.makedirs(d, exist_ok=True)
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(self._cache, fh, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def key(self, workload: dict) -> str:
        return json.dumps({"device": self.device(), "library": self.library(), **workload}, sort_keys=True)

    def choose(self, workload: dict, candidates: list, run: Callable[[dict], Any],
               verify: Optional[Callable[[dict, Any, Any], bool]] = None) -> dict:
        """The fastest of `candidates` (dicts) for `workload` whose answer passes `verify`;
        run(candidate) does one step and returns its answer; verify(candidate, answer,
        reference_answer) compares it with the first candidate's."""
        if not candidates:
            raise ValueError("no candidates")
        k = self.key(workload)
        hit = self._cache.get(k)
        if hit is not None and hit["choice"] in candidates:
            self.last_times = dict(hit["times_ms"])
            self.last_rejected = list(hit.get("rejected", []))
            return dict(hit["choice"])
        times, rejected, reference = {}, [], None
        for idx, cand in enumerate(candidates):
            last = [None]

            def once():
                last[0] = run(cand)

            for _ in range(self.warmup):
                once()
            samples = [self.timer(once) for _ in range(self.repeats)]
            if idx == 0:
                reference = last[0]
            elif verify is not None and not verify(cand, last[0], reference):
                rejected.append(cand)
                continue
            times[json.dumps(cand, sort_keys=True)] = statistics.median(samples)
        ok = [i for i in range(len(candidates)) if json.dumps(candidates[i], sort_keys=True) in times]
        best = min(ok, key=lambda i: (times[json.dumps(candidates[i], sort_keys=True)], i))
        self.last_times = times
        self.last_rejected = rejected
        self._cache[k] = {"choice": candidates[best], "times_ms": times, "rejected": rejected}
        self._save()
        return dict(candidates[best])


def tune_launch_mode(solver, config, prime, candidates=(2, 3), tuner: Optional[Autotuner] = None,
                     workload: Optional[dict] = None) -> int:
    """The `graphs` launch mode for repeated solves of this workload: graph-resident Krylov
    loops (2) or the whole Picard loop as one graph (3).  A mode is only chosen if its
    velocities are bit for bit those of the first candidate's.  prime() sets the initial
    guess of one solve (the solver's inputs are already set)."""
    tuner = tuner or Autotuner()
    wl = {"workload": "ssa solve", "grid": list(solver.shape), "config": config_key(config), **(workload or {})}

    def run(cand):
        solver.set_config(config.copy(graphs=cand["graphs"]))
        prime()
        return solver.solve()

    def same(cand, out, ref):
        import numpy as np
        return out is not None and ref is not None and np.array_equal(np.asarray(out), np.asarray(ref))

    try:
        best = tuner.choose(wl, [{"graphs": int(g)} for g in candidates], run, verify=same)
    finally:
        solver.set_config(config)
    return best["graphs"]


def tune_config_knob(solver, config, prime, name: str, candidates, tuner: Optional[Autotuner] = None,
                     workload: Optional[dict] = None):
    """The value of one launch-shape field of the solver configuration (`name`, e.g.
    mg_post_blocks_per_sm or mg_small_kernel) for repeated solves of this workload.  Such a
    field changes how the kernels are launched, not their arithmetic, so every candidate must
    give the first one's velocities bit for bit; the first candidate is the default."""
    tuner = tuner or Autotuner()
    wl = {"workload": f"ssa solve, {name}", "grid": list(solver.shape), "config": config_key(config),
          **(workload or {})}

    def run(cand):
        solver.set_config(config.copy(**{name: cand[name]}))
        prime()
        return solver.solve()

    def same(cand, out, ref):
        import numpy as np
        return out is not None and ref is not None and np.array_equal(np.asarray(out), np.asarray(ref))

    try:
        best = tuner.choose(wl, [{name: c} for c in candidates], run, verify=same)
    finally:
        solver.set_config(config)
    return best[name]


def tune_mg_post_blocks(solver, config, prime, candidates=(0, 3, 2), tuner: Optional[Autotuner] = None,
                        workload: Optional[dict] = None) -> int:
    """The grid size of the coarse-level multigrid post-smoothing (resident blocks per SM it
    is sized for; 0 = the tile kernels' 4)."""
    return tune_config_knob(solver, config, prime, "mg_post_blocks_per_sm", candidates, tuner, workload)


def tune_small_kernel(solver, config, prime, candidates=(0, 1), tuner: Optional[Autotuner] = None,
                      workload: Optional[dict] = None) -> int:
    """How the multigrid's small levels are cycled: staged from L2 at every step (0) or held
    in the cluster's shared memory (1)."""
    return tune_config_knob(solver, config, prime, "mg_small_kernel", candidates, tuner, workload)


def tune_apply_kernel(solver, config, prime, candidates=(2, 0, 1), tuner: Optional[Autotuner] = None,
                      workload: Optional[dict] = None) -> int:
    """How BiCGStab's FP32 operator apply after each V-cycle runs: its own kernel with plain
    (0) or bulk-copy staged (1) tile loads, or fused into the V-cycle's fine-level pass (2)."""
    return tune_config_knob(solver, config, prime, "mixed_apply_kernel", candidates, tuner, workload)
