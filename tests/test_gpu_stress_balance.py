"""The consumers of the SSA velocity on the GPU (pism_gpu_ssa_stress_balance_3d:
ConstantInColumn, the vertical velocity, the volumetric strain heating) against the oracle
(PISMStressBalance.cc:192-287, 369-499; SSB_Modifier.cc:126-152)."""
import numpy as np
import pytest

from pism_b200 import synthetic as S
from pism_b200.config import GridDesc, SSAConfig, X_PERIODIC
from oracle import ssafd_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pism_b200.ssa import SSAFD, StressBalance  # noqa: E402

RTOL = 1e-12   # FP64 throughout; differences are fused multiply-adds and pow's last bits


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def random_columns(seed, Mx=23, My=19, Mz=13, flow_law="gpbld", periodicity=0):
    """every mask configuration of a 3x3 neighbourhood, thicknesses from 0 to above the
    top level, an enthalpy column per cell"""
    rng = np.random.default_rng(seed)
    z = np.concatenate([[0.0], np.cumsum(rng.uniform(100.0, 400.0, Mz - 1))])
    g = GridDesc(Mx, My, 0.5 * (Mx - 1) * 7e3, 0.5 * (My - 1) * 9e3, periodicity=periodicity, z=z)
    c = SSAConfig(flow_law=flow_law, ssa_enhancement_factor=rng.uniform(0.5, 3.0))
    mask = rng.choice([0.0, 2.0, 3.0, 4.0], size=(Mx, My))
    H = rng.uniform(0.0, z[-1], (Mx, My))
    H[rng.random((Mx, My)) < 0.1] = z[-1]
    H[rng.random((Mx, My)) < 0.1] = 0.0
    bed = rng.uniform(-1000, 1000, (Mx, My))
    f = {"thickness": H, "bed": bed, "surface": bed + H, "mask": mask, "tauc": rng.uniform(1e3, 2e5, (Mx, My)),
         "melange": np.zeros((Mx, My)),
         "enthalpy": rng.uniform(1.0e5, 2.0e5, (Mx, My, Mz)) if flow_law != "isothermal_glen" else None}
    vel = rng.normal(0.0, 3e-6, (Mx, My, 2))
    return g, c, f, vel


def oracle_fields(g, c, f, vel, bmr):
    G, Cc, I = O.from_case(g, c, f)
    u3, v3 = O.constant_in_column(vel, len(G.z))
    return {"u": u3, "v": v3, "w": O.vertical_velocity(G, I, u3, v3, bmr),
            "strain_heating": O.volumetric_strain_heating(G, Cc, I, u3, v3)}


def gpu_fields(g, c, f, vel, bmr, device):
    s = SSAFD(g, c)
    try:
        s.set_inputs(**{k: v for k, v in f.items() if v is not None})
        s.set_initial_guess(vel)
        if device:
            out = s.stress_balance_3d(None if bmr is None else torch.tensor(bmr, device="cuda"), device=True)
            return {k: v.cpu().numpy() for k, v in out.items()}
        return s.stress_balance_3d(bmr)
    finally:
        s.close()


@pytest.mark.parametrize("law,periodicity,bmr,device", [("gpbld", 0, True, False), ("isothermal_glen", 0, False, True),
                                                        ("pb", X_PERIODIC, True, True), ("hooke", 0, False, False)])
def test_columns_match_the_oracle(law, periodicity, bmr, device):
    g, c, f, vel = random_columns(3, flow_law=law, periodicity=periodicity)
    melt = np.random.default_rng(4).uniform(0, 1e-8, (g.Mx, g.My)) if bmr else None
    ref = oracle_fields(g, c, f, vel, melt)
    got = gpu_fields(g, c, f, vel, melt, device)
    np.testing.assert_array_equal(got["u"], ref["u"])
    np.testing.assert_array_equal(got["v"], ref["v"])
    assert relmax(got["w"], ref["w"]) < RTOL
    assert relmax(got["strain_heating"], ref["strain_heating"]) < RTOL
    assert np.all(got["strain_heating"][ref["strain_heating"] == 0.0] == 0.0)


def test_stress_balance_update_after_a_solve():
    """StressBalance::update on a synthetic sheet: the SSA solve, then the 3-D fields from its
    velocity, against the oracle on the same velocity"""
    g0, c, f, _ = S.build_synthetic(61, 4000e3 / 60, seed=2)
    g = GridDesc(g0.Mx, g0.My, g0.Lx, g0.Ly, periodicity=0, z=np.linspace(0.0, 4000.0, 21))
    c = c.copy(pc_type="mg")
    sb = StressBalance(SSAFD(g, c))
    try:
        sb.ssa.set_inputs(**f)
        melt = np.full((g.Mx, g.My), 1e-9)
        sb.set_basal_melt_rate(melt)
        sb.update(fast=False)
        vel = sb.advective_velocity()
        ref = oracle_fields(g, c, f, vel, melt)
        assert relmax(sb.velocity_w(), ref["w"]) < RTOL
        assert relmax(sb.volumetric_strain_heating(), ref["strain_heating"]) < RTOL
        np.testing.assert_array_equal(sb.velocity_u(), ref["u"])
    finally:
        sb.ssa.close()


def test_refuses_without_levels_or_enthalpy():
    g, c, f, vel = random_columns(5)
    s = SSAFD(g, c)
    try:
        s.set_inputs(**{k: v for k, v in f.items() if k != "enthalpy"}, hardness=np.ones((g.Mx, g.My, 2)))
        with pytest.raises(Exception):
            s.stress_balance_3d()
    finally:
        s.close()


def test_two_levels_and_the_top_level():
    """Mz = 2 (the fewest the strain heating's one-sided z difference needs) with thicknesses
    at 0 and at the top level: kBelowHeight is 0 for both, so only level 0 heats"""
    g, c, f, vel = random_columns(9, Mz=2, flow_law="isothermal_glen")
    f = dict(f, thickness=np.where(np.arange(g.Mx)[:, None] % 2 == 0, 0.0, g.z[-1]) * np.ones((g.Mx, g.My)))
    ref = oracle_fields(g, c, f, vel, None)
    got = gpu_fields(g, c, f, vel, None, device=False)
    assert relmax(got["w"], ref["w"]) < RTOL
    assert relmax(got["strain_heating"], ref["strain_heating"]) < RTOL
    assert np.all(got["strain_heating"][..., 1] == 0.0)
