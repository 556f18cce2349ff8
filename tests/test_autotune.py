"""The autotuner's choice, timing protocol and cache (CPU, with an injected timer)."""
import json

import pytest

from pism_b200.autotune import Autotuner


class FakeClock:
    """Timer whose reading is the cost the candidate run declared."""

    def __init__(self):
        self.cost = 0.0
        self.calls = 0

    def __call__(self, run):
        run()
        self.calls += 1
        return self.cost


def make(tmp_path, repeats=3, warmup=1):
    clock = FakeClock()
    tuner = Autotuner(str(tmp_path / "tune.json"), repeats=repeats, warmup=warmup, timer=clock,
                      device=lambda: "B200-fake", library=lambda: "lib-a")
    return tuner, clock


def test_picks_the_fastest_and_counts_runs(tmp_path):
    tuner, clock = make(tmp_path)
    costs = {1: 5.0, 2: 3.0, 4: 2.0, 8: 2.5}
    runs = []

    def run(c):
        runs.append(c["streams"])
        clock.cost = costs[c["streams"]]

    best = tuner.choose({"w": 1}, [{"streams": s} for s in (1, 2, 4, 8)], run)
    assert best == {"streams": 4}
    assert len(runs) == 4 * (1 + 3) and clock.calls == 4 * 3   # warm-up untimed, repeats timed
    assert tuner.last_times[json.dumps({"streams": 4})] == 2.0


def test_median_of_repeats_and_ties_go_to_the_first(tmp_path):
    tuner, clock = make(tmp_path, repeats=3, warmup=0)
    seq = iter([10.0, 1.0, 10.0,   # a: median 10 despite one fast sample
                4.0, 4.0, 4.0,     # b: 4
                4.0, 4.0, 4.0])    # c: 4, tie with b
    def run(c):
        clock.cost = next(seq)
    assert tuner.choose({"w": 2}, [{"x": "a"}, {"x": "b"}, {"x": "c"}], run) == {"x": "b"}


def test_cache_is_reused_and_keyed_by_device_and_workload(tmp_path):
    tuner, clock = make(tmp_path)
    clock.cost = 1.0
    cands = [{"streams": 1}, {"streams": 2}]
    tuner.choose({"grid": [401, 401]}, cands, lambda c: None)
    n = clock.calls
    again = Autotuner(str(tmp_path / "tune.json"), timer=clock, device=lambda: "B200-fake", library=lambda: "lib-a")
    assert again.choose({"grid": [401, 401]}, cands, lambda c: pytest.fail("ran despite the cache")) == {"streams": 1}
    assert clock.calls == n
    other_dev = Autotuner(str(tmp_path / "tune.json"), timer=clock, device=lambda: "other", library=lambda: "lib-a")
    other_dev.choose({"grid": [401, 401]}, cands, lambda c: None)
    assert clock.calls > n
    # a cached choice that is no longer a candidate is tuned again
    m = clock.calls
    again.choose({"grid": [401, 401]}, [{"streams": 4}], lambda c: None)
    assert clock.calls > m


def test_rejects_bad_arguments(tmp_path):
    with pytest.raises(ValueError):
        Autotuner(repeats=0)
    tuner, _ = make(tmp_path)
    with pytest.raises(ValueError):
        tuner.choose({"w": 3}, [], lambda c: None)


def test_another_library_build_is_tuned_again(tmp_path):
    """the cache key holds the library's fingerprint: a choice made with other kernels is not reused"""
    tuner, clock = make(tmp_path)
    clock.cost = 1.0
    cands = [{"streams": 1}, {"streams": 2}]
    tuner.choose({"grid": [401, 401]}, cands, lambda c: None)
    n = clock.calls
    rebuilt = Autotuner(str(tmp_path / "tune.json"), timer=clock, device=lambda: "B200-fake", library=lambda: "lib-b")
    rebuilt.choose({"grid": [401, 401]}, cands, lambda c: None)
    assert clock.calls > n


def test_a_candidate_with_another_answer_is_never_chosen(tmp_path):
    """verify(candidate, answer, reference answer): the first candidate's answer is the
    reference; a faster candidate whose answer differs is rejected and recorded"""
    tuner, clock = make(tmp_path, repeats=1, warmup=0)
    costs = {"a": 5.0, "b": 1.0, "c": 3.0}
    answers = {"a": 42, "b": 41, "c": 42}

    def run(c):
        clock.cost = costs[c["x"]]
        return answers[c["x"]]

    best = tuner.choose({"w": 9}, [{"x": "a"}, {"x": "b"}, {"x": "c"}], run,
                        verify=lambda cand, out, ref: out == ref)
    assert best == {"x": "c"}
    assert tuner.last_rejected == [{"x": "b"}]
    # the cached entry keeps the rejection
    again = Autotuner(str(tmp_path / "tune.json"), timer=clock, device=lambda: "B200-fake", library=lambda: "lib-a")
    assert again.choose({"w": 9}, [{"x": "a"}, {"x": "b"}, {"x": "c"}], lambda c: pytest.fail("ran")) == {"x": "c"}
    assert again.last_rejected == [{"x": "b"}]


def test_mg_post_blocks_through_the_solver_interface(tmp_path):
    """tune_mg_post_blocks: the launch shape changes the time, never the answer; a candidate
    whose velocities differ from the default's is rejected"""
    import numpy as np
    from pism_b200.autotune import tune_mg_post_blocks
    from pism_b200.config import SSAConfig
    tuner, clock = make(tmp_path, repeats=1, warmup=0)

    class Solver:
        shape = (801, 801)

        def __init__(self):
            self.cfg = None

        def set_config(self, c):
            self.cfg = c

        def solve(self):
            b = self.cfg.mg_post_blocks_per_sm
            clock.cost = {0: 130.0, 3: 120.0, 2: 110.0}[b]
            return np.ones(4) * (2.0 if b == 2 else 1.0)   # the 2-block run "differs"

    s = Solver()
    base = SSAConfig(pc_type="mg", precision="mixed")
    assert tune_mg_post_blocks(s, base, prime=lambda: None, tuner=tuner) == 3
    assert s.cfg is base


def test_launch_mode_through_the_solver_interface(tmp_path):
    """tune_launch_mode times solves under each `graphs` value and restores the config."""
    from pism_b200.autotune import tune_launch_mode
    from pism_b200.config import SSAConfig
    tuner, clock = make(tmp_path, repeats=1, warmup=0)

    class Solver:
        shape = (801, 801)

        def __init__(self):
            self.cfg = None
            self.log = []

        def set_config(self, c):
            self.cfg = c

        def solve(self):
            self.log.append(self.cfg.graphs)
            clock.cost = {2: 130.0, 3: 120.0}[self.cfg.graphs]
            return [1.0, 2.0]

    s = Solver()
    base = SSAConfig(pc_type="mg", precision="mixed")
    assert tune_launch_mode(s, base, prime=lambda: None, tuner=tuner) == 3
    assert s.log == [2, 3] and s.cfg is base


def test_small_kernel_through_the_solver_interface(tmp_path):
    """tune_small_kernel: both small-level cycles give the same bits; the faster is chosen"""
    import numpy as np
    from pism_b200.autotune import tune_small_kernel
    from pism_b200.config import SSAConfig
    tuner, clock = make(tmp_path, repeats=1, warmup=0)

    class Solver:
        shape = (401, 401)
        cfg = None

        def set_config(self, c):
            self.cfg = c

        def solve(self):
            clock.cost = {0: 50.0, 1: 48.0}[self.cfg.mg_small_kernel]
            return np.ones(3)

    s = Solver()
    base = SSAConfig(pc_type="mg")
    assert tune_small_kernel(s, base, prime=lambda: None, tuner=tuner) == 1
    assert s.cfg is base


def test_apply_kernel_through_the_solver_interface(tmp_path):
    """the three BiCGStab apply kernels are timed like any other knob, the fastest chosen and
    the caller's configuration left as it was"""
    import numpy as np
    from pism_b200.autotune import tune_apply_kernel
    from pism_b200.config import SSAConfig
    tuner, clock = make(tmp_path, repeats=1, warmup=0)

    class Solver:
        shape = (801, 801)
        cfg = None

        def set_config(self, c):
            self.cfg = c

        def solve(self):
            clock.cost = {0: 230.0, 1: 228.0, 2: 200.0}[self.cfg.mixed_apply_kernel]
            return np.ones(3)

    s = Solver()
    base = SSAConfig(pc_type="mg", precision="mixed")
    assert tune_apply_kernel(s, base, prime=lambda: None, tuner=tuner) == 2
    assert s.cfg is base
