"""The bench's bookkeeping on CPU: multigrid level sizes (2 x 2 aggregation down to at most
4 x 4 cells, as mg_plan does) and the algorithmic bytes of one Krylov iteration."""
import importlib.util
import os

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_model", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_levels_of_the_801_grid():
    b = _bench()
    assert b.mg_levels(801) == [401 ** 2, 201 ** 2, 101 ** 2, 51 ** 2, 26 ** 2, 13 ** 2, 7 ** 2, 4 ** 2]
    assert b.mg_levels(4) == []
    assert b.mg_levels(5) == [9]


def test_iteration_bytes():
    """per fine cell: p 32 + x 72 + restricts 40 + 48, then the fused post + apply 64 + 64
    (apply_kernel 2) or posts 48 + 56 and applies 40 + 48 (0, 1); per V-cycle 16 B per
    level-1 cell and 344 B per coarse cell"""
    b = _bench()
    N0, lev = 801 ** 2, b.mg_levels(801)
    coarse = 2 * (16 * lev[0] + 344 * sum(lev))
    fused = 320 * N0 + coarse
    assert b.iteration_bytes(801, "mixed") == fused
    assert b.iteration_bytes(801, "mixed", 0) == b.iteration_bytes(801, "mixed", 1) == 384 * N0 + coarse
    assert b.iteration_bytes(801, "fp64") > b.iteration_bytes(801, "mixed", 0)
    assert 350e6 < fused < 365e6


def test_fast_config_keeps_the_accepted_tolerance():
    b = _bench()
    from pism_b200.config import SSAConfig
    c = b.fast_config(SSAConfig())
    assert c.ksp_rtol == 1e-6 and c.ksp_rtol_adaptive and c.precision == "mixed"
    assert c.ksp_rtol_max >= c.ksp_rtol
