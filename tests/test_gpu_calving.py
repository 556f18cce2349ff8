"""The strain rates, 2-D stresses and eigen-calving on the GPU (pism_gpu_ssa_strain_rates,
pism_gpu_ssa_eigen_calving, pism_gpu_ssa_eigen_calving_max_timestep) against the oracle
(ShallowStressBalance.cc:224-386; PISMEigenCalving.cc:77-493)."""
import numpy as np
import pytest

from pism_b200.config import GridDesc, SSAConfig
from oracle import ssafd_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pism_b200.ssa import SSAFD, StressBalance, EigenCalving  # noqa: E402

RTOL_POW = 1e-13   # the stresses go through pow(), whose last bit may differ from the host's


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def random_front(seed, Mx=41, My=37, d=5e3):
    """a mostly floating mask with every kind of neighbourhood, a spreading velocity with
    noise (so that both principal strain rates are often positive), Href and thickness"""
    rng = np.random.default_rng(seed)
    g = GridDesc(Mx, My, 0.5 * (Mx - 1) * d, 0.5 * (My - 1) * d)
    mask = rng.choice([0.0, 2.0, 3.0, 4.0], p=[0.1, 0.1, 0.5, 0.3], size=(Mx, My))
    H = np.where((mask == 2) | (mask == 3), rng.uniform(100.0, 800.0, (Mx, My)), 0.0)
    x = np.arange(Mx)[:, None] * d * np.ones((1, My))
    y = np.arange(My)[None, :] * d * np.ones((Mx, 1))
    vel = np.stack([1e-9 * x, 7e-10 * y], axis=-1) + rng.normal(0.0, 2e-6, (Mx, My, 2))
    Href = np.where(mask == 4, rng.uniform(0.0, 50.0, (Mx, My)), 0.0)
    f = {"thickness": H, "bed": np.full((Mx, My), -2000.0), "surface": 0.1 * H, "mask": mask,
         "tauc": np.full((Mx, My), 1e5), "melange": np.zeros((Mx, My))}
    return g, f, vel, Href


def handle(g, f, vel, config=None):
    s = SSAFD(g, config or SSAConfig())
    s.set_inputs(**f)
    s.set_initial_guess(vel)
    return s


@pytest.mark.parametrize("device,own_mask", [(False, False), (True, True), (False, True)])
def test_strain_rates_and_stresses_match_the_oracle(device, own_mask):
    g, f, vel, _ = random_front(1)
    mask = f["mask"]
    if own_mask:   # a different mask than the inputs' one
        mask = np.where(np.random.default_rng(2).random(mask.shape) < 0.2, 4.0, mask)
    G = O.Grid(g.Mx, g.My, g.Lx, g.Ly)
    ref_e = O.principal_strain_rates(G, mask, vel)
    ref_s = O.deviatoric_stresses_2d(G, O.Config(), mask, vel)
    s = handle(g, f, vel)
    try:
        arg = (torch.tensor(mask, device="cuda") if device else mask) if own_mask else None
        out = s.strain_rates(arg, device=device)
    finally:
        s.close()
    e = out["edot"].cpu().numpy() if device else out["edot"]
    st = out["stresses"].cpu().numpy() if device else out["stresses"]
    np.testing.assert_array_equal(e, ref_e)
    assert relmax(st, ref_s) < RTOL_POW
    assert np.all(st[O.m_ice_free(O.as_int(mask))] == 0.0)


def test_stress_balance_names():
    g, f, vel, _ = random_front(3)
    s = handle(g, f, vel)
    try:
        sb = StressBalance(s)
        G = O.Grid(g.Mx, g.My, g.Lx, g.Ly)
        np.testing.assert_array_equal(sb.compute_2D_principal_strain_rates(), O.principal_strain_rates(G, f["mask"], vel))
        assert relmax(sb.compute_2D_stresses(), O.deviatoric_stresses_2d(G, O.Config(), f["mask"], vel)) < RTOL_POW
    finally:
        s.close()


@pytest.mark.parametrize("seed,K,device", [(4, 3e13, False), (5, 1e14, True), (6, 1e12, False)])
def test_eigen_calving_matches_the_oracle(seed, K, device):
    g, f, vel, Href = random_front(seed)
    G = O.Grid(g.Mx, g.My, g.Lx, g.Ly)
    dt = 1e7
    ref_m, ref_href, ref_h = O.eigen_calving(G, f["mask"], Href, f["thickness"], vel, dt, K)
    s = handle(g, f, vel)
    try:
        t = (lambda a: torch.tensor(a, device="cuda")) if device else (lambda a: a)
        out = s.eigen_calving(dt, K, t(f["mask"]), t(Href), t(f["thickness"]))
    finally:
        s.close()
    got = {k: (v.cpu().numpy() if device else v) for k, v in out.items()}
    np.testing.assert_array_equal(got["mask"], ref_m)
    np.testing.assert_array_equal(got["Href"], ref_href)
    np.testing.assert_array_equal(got["thickness"], ref_h)
    # the case calves: cells were cut and Href changed
    assert np.any(ref_m != f["mask"]) and np.any(ref_href != Href)


def test_narrow_tongues_in_the_reference_order():
    """no calving (K = 0): only remove_narrow_tongues acts, on tongues pointing both ways in x
    and y, where the reference's loop order decides how much of a tongue goes"""
    Mx, My = 24, 22
    F, OC = O.MASK_FLOATING, O.MASK_ICE_FREE_OCEAN
    M = np.full((Mx, My), float(OC))
    M[:3, :] = F
    M[3:7, 6] = F        # east-pointing
    M[19:, :] = F
    M[14:19, 12] = F     # west-pointing
    M[8:12, 0:3] = F
    M[9, 3:8] = F        # north-pointing
    M[8:12, 19:] = F
    M[10, 14:19] = F     # south-pointing
    M[15, 3] = 2.0       # a grounded pair in ice-free ocean
    M[16, 3] = 2.0
    H = np.where(M != OC, 300.0, 0.0)
    g = GridDesc(Mx, My, 0.5 * (Mx - 1) * 5e3, 0.5 * (My - 1) * 5e3)
    G = O.Grid(Mx, My, g.Lx, g.Ly)
    vel = np.zeros((Mx, My, 2))
    ref_m, _, ref_h = O.eigen_calving(G, M, np.zeros((Mx, My)), H, vel, 1e7, 0.0)
    f = {"thickness": H, "bed": np.full((Mx, My), -2000.0), "surface": 0.1 * H, "mask": M,
         "tauc": np.full((Mx, My), 1e5)}
    s = handle(g, f, vel)
    try:
        sb = StressBalance(s)
        ec = EigenCalving(sb, K=0.0)
        m, href, h = M.copy(), np.zeros((Mx, My)), H.copy()
        ec.update(1e7, m, href, h)
    finally:
        s.close()
    np.testing.assert_array_equal(m, ref_m)
    np.testing.assert_array_equal(h, ref_h)
    assert np.count_nonzero(ref_m != M) >= 5


@pytest.mark.parametrize("device", [False, True])
def test_max_timestep_matches_the_oracle(device):
    g, f, vel, _ = random_front(7)
    G = O.Grid(g.Mx, g.My, g.Lx, g.Ly)
    K = 3e13
    dt, rmax, rmean, count = O.eigen_calving_max_timestep(G, f["mask"], vel, K)
    s = handle(g, f, vel)
    try:
        ec = EigenCalving(StressBalance(s), K=K, restrict_timestep=True)
        got = ec.max_timestep(torch.tensor(f["mask"], device="cuda") if device else f["mask"])
        r = ec.last_rates
        assert EigenCalving(StressBalance(s), K=K).max_timestep(f["mask"]) is None
    finally:
        s.close()
    assert count > 0 and r["count"] == count
    assert r["max_rate"] == rmax
    assert r["mean_rate"] == pytest.approx(rmean, rel=1e-12)
    assert got == pytest.approx(dt, rel=1e-14)
