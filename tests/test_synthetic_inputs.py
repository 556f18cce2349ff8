"""The seeded synthetic workloads (CPU): the 801 x 801 benchmark sheet and the ensemble
members are drawn from the distributions they stand in for — bed from a Gaussian random
field (mean -300 m, std 800 m, correlation length 100 km), thickness in [0, 4000] m with the
floating mask from flotation at sea level 0 (densities 910 / 1028), lognormal tau_c
(median 50 kPa, sigma 1), hardness from uniform -10 C ice; ensemble members with ice
temperature in [-20, -2] C and tau_c median in [20, 200] kPa."""
import importlib.util
import math
import os

import numpy as np
import pytest

from pism_b200 import synthetic as S
from pism_b200.config import SSAConfig

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def sheet():
    return S.build_synthetic(801, 5.0e3, seed=0)


def lag_correlation(f, lag):
    a, b = f[:-lag], f[lag:]
    return float(np.mean((a - a.mean()) * (b - b.mean())) / (a.std() * b.std()))


def test_random_field_statistics():
    """exp(-r^2 / l^2) covariance, unit variance: correlation e^-1 at lag l (100 km = 20 cells)."""
    rng = np.random.Generator(np.random.PCG64(3))
    f = S._grf(rng, 801, 5.0e3, 100.0e3)
    assert abs(f.mean()) < 1e-12 and abs(f.std() - 1.0) < 1e-12
    for lag, want in ((10, math.exp(-0.25)), (20, math.exp(-1.0)), (40, math.exp(-4.0))):
        got = 0.5 * (lag_correlation(f, lag) + lag_correlation(f.T, lag))
        assert got == pytest.approx(want, abs=0.06), lag


def test_bed_distribution(sheet):
    g, c, f, meta = sheet
    L = 800 * 5.0e3
    x = np.arange(801) * 5.0e3
    X, Y = np.meshgrid(x, x, indexing="ij")
    dist = np.minimum(np.minimum(X, L - X), np.minimum(Y, L - Y))
    inner = f["bed"][dist >= meta["border"]]          # untouched by the deep-ocean border taper
    assert inner.mean() == pytest.approx(-300.0, abs=120.0)
    assert inner.std() == pytest.approx(800.0, rel=0.2)
    edge = f["bed"][dist == 0]
    assert np.all(edge == -3000.0)


def test_thickness_mask_and_surface(sheet):
    g, c, f, _ = sheet
    H, bed, mask, srf = f["thickness"], f["bed"], f["mask"], f["surface"]
    assert H.min() >= 0.0 and H.max() <= 4000.0
    assert set(np.unique(mask)) <= {0.0, 2.0, 3.0, 4.0}
    alpha = 1.0 - c.ice_density / c.sea_water_density
    assert c.ice_density == 910.0 and c.sea_water_density == 1028.0 and c.sea_level == 0.0
    floating = alpha * H > bed + H + c.mask_is_floating_thickness_standard
    icy = H >= c.mask_icefree_thickness_standard   # GeometryCalculator's ice-free threshold
    np.testing.assert_array_equal(mask == 3.0, floating & icy)
    np.testing.assert_array_equal(mask == 2.0, ~floating & icy)
    np.testing.assert_allclose(srf, np.where(floating, alpha * H, bed + H))
    assert (mask == 2.0).sum() > 1000 and (mask == 3.0).sum() > 100   # grounded ice and shelves


def test_tauc_is_lognormal_with_median_50kpa(sheet):
    g, c, f, _ = sheet
    z = np.log(f["tauc"] / 50.0e3)
    assert abs(z.mean()) < 1e-12 and abs(z.std() - 1.0) < 1e-12
    assert np.median(f["tauc"]) == pytest.approx(50.0e3, rel=0.15)


def test_hardness_from_minus_ten_degrees(sheet):
    g, c, f, _ = sheet
    assert c.flow_law == "isothermal_glen"
    ref = SSAConfig()
    T = 273.15 - 10.0   # at the Paterson-Budd critical temperature: the warm branch
    A = ref.Paterson_Budd_A_warm * math.exp(-ref.Paterson_Budd_Q_warm / (ref.ideal_gas_constant * T))
    assert c.ice_softness == pytest.approx(A, rel=1e-15)
    assert c.ssafd_relative_convergence == 1e-4 and c.ksp_rtol == 1e-8


def test_seeded_and_reproducible():
    a = S.build_synthetic(65, 62.5e3, seed=4)[2]
    b = S.build_synthetic(65, 62.5e3, seed=4)[2]
    d = S.build_synthetic(65, 62.5e3, seed=5)[2]
    for k in ("thickness", "bed", "tauc"):
        np.testing.assert_array_equal(a[k], b[k])
        assert not np.array_equal(a[k], d[k])


def test_ensemble_members():
    spec = importlib.util.spec_from_file_location("bench_members", os.path.join(REPO, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    draws = [bench.ensemble_member(q, M=33)[3] for q in range(8)]
    Ts = [d["T"] for d in draws]
    meds = [d["tauc_median"] for d in draws]
    assert all(-20.0 <= t <= -2.0 for t in Ts) and all(20e3 <= m <= 200e3 for m in meds)
    assert len(set(Ts)) == 8 and len(set(meds)) == 8
    g, c, f, d = bench.ensemble_member(0, M=33)
    assert np.median(f["tauc"]) == pytest.approx(d["tauc_median"], rel=0.6)
    assert c.ice_softness == pytest.approx(S.paterson_budd_softness(273.15 + d["T"], c), rel=1e-15)
