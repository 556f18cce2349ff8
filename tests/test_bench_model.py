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
    b = _bench()
    N0, lev = 801 ** 2, b.mg_levels(801)
    mixed = 200 * N0 + 2 * (90 * N0 + 16 * lev[0] + 344 * sum(lev))
    assert b.iteration_bytes(801, "mixed") == mixed
    assert b.iteration_bytes(801, "fp64") > mixed
    assert 390e6 < mixed < 400e6


def test_fast_config_keeps_the_accepted_tolerance():
    b = _bench()
    from pism_b200.config import SSAConfig
    c = b.fast_config(SSAConfig())
    assert c.ksp_rtol == 1e-6 and c.ksp_rtol_adaptive and c.precision == "mixed"
    assert c.ksp_rtol_max >= c.ksp_rtol
