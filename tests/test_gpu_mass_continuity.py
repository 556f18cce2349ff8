"""The explicit mass-continuity step on the GPU (pism_gpu_ssa_mass_continuity_step) against
the oracle (IceModel::massContExplicitStep, iMgeometry.cc:497-819; updateSurfaceElevationAndMask,
iMgeometry.cc:56-68)."""
import numpy as np
import pytest

from pism_b200 import synthetic as S
from pism_b200.config import GridDesc, SSAConfig, X_PERIODIC
from oracle import ssafd_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pism_b200.ssa import SSAFD  # noqa: E402

RTOL = 1e-12   # FP64; the GPU contracts products into fused multiply-adds


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def random_step(seed, Mx=29, My=23, dirichlet=False, periodicity=0):
    """every mask neighbourhood, thin ice that the step drives below zero, Dirichlet cells"""
    rng = np.random.default_rng(seed)
    g = GridDesc(Mx, My, 0.5 * (Mx - 1) * 5e3, 0.5 * (My - 1) * 6e3, periodicity=periodicity)
    c = SSAConfig(ssa_dirichlet_bc=dirichlet)
    mask = rng.choice([0.0, 2.0, 3.0, 4.0], size=(Mx, My))
    H = np.where((mask == 2) | (mask == 3), rng.uniform(1.0, 2000.0, (Mx, My)), rng.uniform(0.0, 5.0, (Mx, My)))
    bed = rng.uniform(-1000.0, 1000.0, (Mx, My))
    f = {"thickness": H, "bed": bed, "surface": bed + H, "mask": mask, "tauc": np.full((Mx, My), 1e4),
         "melange": np.zeros((Mx, My))}
    if dirichlet:
        f["bc_mask"] = (rng.random((Mx, My)) < 0.1).astype(float)
        f["bc_values"] = rng.normal(0.0, 1e-5, (Mx, My, 2))
    vel = rng.normal(0.0, 1e-5, (Mx, My, 2))
    cmb = rng.normal(0.0, 2e-5, (Mx, My))
    bmr = rng.uniform(0.0, 5e-8, (Mx, My))
    area = rng.uniform(0.9, 1.1, (Mx, My)) * g.dx * g.dy
    return g, c, f, vel, cmb, bmr, area


def oracle_step(g, c, f, vel, dt, cmb, bmr, area):
    G, Cc, I = O.from_case(g, c, f)
    Hn, fdiv, tot = O.mass_continuity_step(G, Cc, I, vel, dt, cmb, bmr, area)
    mask, surface = O.geometry_mask_surface(Cc, I.bed, Hn)
    return {"thickness": Hn, "flux_divergence": fdiv, "mask": mask, "surface": surface, "totals": tot}


def gpu_step(g, c, f, vel, dt, cmb, bmr, area, device):
    s = SSAFD(g, c)
    try:
        s.set_inputs(**f)
        s.set_initial_guess(vel)
        if device:
            t = lambda a: None if a is None else torch.tensor(a, device="cuda")
            out = s.mass_continuity_step(dt, t(cmb), t(bmr), t(area))
            return {k: (v if k == "totals" else v.cpu().numpy()) for k, v in out.items()}
        return s.mass_continuity_step(dt, cmb, bmr, area)
    finally:
        s.close()


@pytest.mark.parametrize("dirichlet,periodicity,melt,device", [(False, 0, True, False), (True, 0, True, True),
                                                               (False, X_PERIODIC, False, True)])
def test_step_matches_the_oracle(dirichlet, periodicity, melt, device):
    g, c, f, vel, cmb, bmr, area = random_step(7, dirichlet=dirichlet, periodicity=periodicity)
    dt = 5.0e6
    b = bmr if melt else None
    ref = oracle_step(g, c, f, vel, dt, cmb, b, area)
    got = gpu_step(g, c, f, vel, dt, cmb, b, area, device)
    assert relmax(got["thickness"], ref["thickness"]) < RTOL
    assert relmax(got["flux_divergence"], ref["flux_divergence"]) < RTOL
    assert relmax(got["surface"], ref["surface"]) < RTOL
    np.testing.assert_array_equal(got["mask"], ref["mask"])
    assert np.any(ref["thickness"] == 0.0) and np.all(got["thickness"] >= 0.0)
    for k, v in ref["totals"].items():
        assert got["totals"][k] == pytest.approx(v, rel=1e-11, abs=1e-6), k


def test_step_after_an_ssa_solve():
    """one model step on a synthetic sheet: the SSA solve, then the mass transport from its
    velocity, with the default cell area (dx dy)"""
    g, c, f, _ = S.build_synthetic(61, 4000e3 / 60, seed=4)
    s = SSAFD(g, c.copy(pc_type="mg"))
    try:
        s.set_inputs(**f)
        vel = s.solve()
        cmb = np.full((61, 61), 1e-5)
        out = s.mass_continuity_step(3.15e7, cmb)
    finally:
        s.close()
    ref = oracle_step(g, c, f, vel, 3.15e7, cmb, None, None)
    assert relmax(out["thickness"], ref["thickness"]) < RTOL
    np.testing.assert_array_equal(out["mask"], ref["mask"])


def test_a_zero_step_changes_nothing():
    """dt = 0: the thickness is returned unchanged (no cell goes negative) and every total is 0"""
    g, c, f, vel, cmb, bmr, area = random_step(11, dirichlet=True)
    out = gpu_step(g, c, f, vel, 0.0, cmb, bmr, area, device=False)
    np.testing.assert_array_equal(out["thickness"], f["thickness"])
    assert all(v == 0.0 for v in out["totals"].values())
