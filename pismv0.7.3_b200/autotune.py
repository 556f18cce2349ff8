"""The project's autotuner: choose the fastest launch configuration of a workload by timing
the candidates on the device, and remember the choice per (device, workload).

    tuner = Autotuner("tuning.json")
    best = tuner.choose({"workload": "ensemble", "grid": [401, 401]},
                        [{"streams": 1}, {"streams": 2}, {"streams": 4}, {"streams": 8}],
                        lambda cand: s.solve_batch(sample, net=net, streams=cand["streams"]))

Each candidate runs `warmup` untimed times, then `repeats` timed times; its time is the
median.  Timing is done with CUDA events on the current stream around the call, with a
synchronize on both sides (the solver calls return with their work complete).  Ties go to
the earlier candidate, so list the default first.  The cache is a JSON file keyed by the
device name and the workload description; a cached choice is returned without running
anything, as long as it is still one of the candidates.
"""
from __future__ import annotations

import json
import os
import statistics
from typing import Callable, Optional


def cuda_event_timer(run: Callable[[], None]) -> float:
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


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, repeats: int = 3, warmup: int = 1,
                 timer: Callable[[Callable[[], None]], float] = cuda_event_timer,
                 device: Optional[Callable[[], str]] = None):
        if repeats < 1 or warmup < 0:
            raise ValueError("repeats >= 1 and warmup >= 0")
        self.cache_path = cache_path
        self.repeats = repeats
        self.warmup = warmup
        self.timer = timer
        self.device = device or device_name
        self.last_times: dict[str, float] = {}
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
        return json.dumps({"device": self.device(), **workload}, sort_keys=True)

    def choose(self, workload: dict, candidates: list, run: Callable[[dict], None]) -> dict:
        """The fastest of `candidates` (dicts) for `workload`; run(candidate) does one step."""
        if not candidates:
            raise ValueError("no candidates")
        k = self.key(workload)
        hit = self._cache.get(k)
        if hit is not None and hit["choice"] in candidates:
            self.last_times = dict(hit["times_ms"])
            return dict(hit["choice"])
        times = {}
        for cand in candidates:
            for _ in range(self.warmup):
                run(cand)
            samples = [self.timer(lambda: run(cand)) for _ in range(self.repeats)]
            times[json.dumps(cand, sort_keys=True)] = statistics.median(samples)
        best = min(range(len(candidates)), key=lambda i: (times[json.dumps(candidates[i], sort_keys=True)], i))
        self.last_times = times
        self._cache[k] = {"choice": candidates[best], "times_ms": times}
        self._save()
        return dict(candidates[best])


def tune_ensemble_streams(solver, members, net=None, stride: int = 1, candidates=(1, 2, 4, 8),
                          tuner: Optional[Autotuner] = None, workload: Optional[dict] = None) -> int:
    """Members in flight for pism_gpu_ssa_solve_batch_concurrent on this workload, timed on
    `members` (a sample of the ensemble, at least max(candidates) of them)."""
    tuner = tuner or Autotuner()
    wl = {"workload": "ssa ensemble", "grid": list(solver.shape), "members": len(members), **(workload or {})}
    best = tuner.choose(wl, [{"streams": int(c)} for c in candidates],
                        lambda cand: solver.solve_batch([dict(m) for m in members], net=net, stride=stride,
                                                        streams=cand["streams"]))
    return best["streams"]


def tune_launch_mode(solver, config, prime, candidates=(2, 3), tuner: Optional[Autotuner] = None,
                     workload: Optional[dict] = None) -> int:
    """The `graphs` launch mode for repeated solves of this workload: graph-resident Krylov
    loops (2) or the whole Picard loop as one graph (3), both giving the same answers.
    prime() sets the initial guess of one solve (the solver's inputs are already set)."""
    tuner = tuner or Autotuner()
    wl = {"workload": "ssa solve", "grid": list(solver.shape), "precision": config.precision,
          "pc": config.pc_type, **(workload or {})}

    def run(cand):
        solver.set_config(config.copy(graphs=cand["graphs"]))
        prime()
        solver.solve()

    try:
        best = tuner.choose(wl, [{"graphs": int(g)} for g in candidates], run)
    finally:
        solver.set_config(config)
    return best["graphs"]
