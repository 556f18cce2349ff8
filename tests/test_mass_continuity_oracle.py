"""The oracle's restatement of the explicit mass-continuity step (IceModel::massContExplicitStep,
iMgeometry.cc:497-819) against closed-form answers and its own conservation law: the
reference's tests print no vectors for it, so it is pinned by fields whose fluxes are exact."""
import numpy as np
import pytest

from oracle import ssafd_oracle as O


def grid(Mx=12, My=10):
    return O.Grid(Mx, My, 0.5 * (Mx - 1) * 5e3, 0.5 * (My - 1) * 4e3)


def inputs(G, H, mask, bc_mask=None, bc_values=None):
    shape = (G.Mx, G.My)
    return O.Inputs(thickness=H, surface=np.zeros(shape), bed=np.zeros(shape), mask=mask, tauc=np.zeros(shape),
                    bc_mask=bc_mask, bc_values=bc_values)


def test_face_velocities_follow_the_four_mask_cases():
    G = grid()
    mask = np.full((G.Mx, G.My), 2.0)
    mask[6:, :] = 0.0   # ice-free bedrock from row 6
    rng = np.random.default_rng(0)
    vel = rng.normal(size=(G.Mx, G.My, 2))
    f = O.cell_interface_velocities(O.Config(), inputs(G, np.ones((G.Mx, G.My)), mask), vel)
    u = vel[..., 0]
    assert f["e"][3, 4] == pytest.approx(0.5 * (u[3, 4] + u[4, 4]))   # both icy
    assert f["e"][5, 4] == u[5, 4]                                     # icy, ice-free east
    assert f["w"][6, 4] == u[5, 4]                                     # ice-free, icy west
    assert f["e"][8, 4] == 0.0                                         # both ice-free


def test_dirichlet_locations_use_their_prescribed_velocity():
    G = grid()
    mask = np.full((G.Mx, G.My), 2.0)
    bc = np.zeros((G.Mx, G.My))
    bc[4, 3] = bc[5, 3] = 1.0
    bcv = np.zeros((G.Mx, G.My, 2))
    bcv[4, 3], bcv[5, 3] = (1.0, 2.0), (3.0, 4.0)
    vel = np.full((G.Mx, G.My, 2), 10.0)
    cfg = O.Config(ssa_dirichlet_bc=True)
    f = O.cell_interface_velocities(cfg, inputs(G, np.ones((G.Mx, G.My)), mask, bc, bcv), vel)
    assert f["e"][4, 3] == 0.5 * (1.0 + 3.0)   # both B.C. locations
    assert f["n"][4, 3] == 2.0                 # at a B.C. location
    assert f["e"][3, 3] == 1.0                 # next to one
    assert f["e"][2, 3] == 10.0                # elsewhere: the regular average


def test_upwinded_divergence_of_a_ramp():
    """u = U > 0 everywhere on icy cells, H = h0 + a i: the upwinded divergence is
    U (H_i - H_{i-1}) / dx = U a / dx away from the periodic seam"""
    G = grid()
    U, h0, a = 3e-6, 500.0, 7.0
    i = np.arange(G.Mx)[:, None] * np.ones((1, G.My))
    H = h0 + a * i
    vel = np.zeros((G.Mx, G.My, 2))
    vel[..., 0] = U
    dt = 1e6
    Hn, fdiv, _ = O.mass_continuity_step(G, O.Config(), inputs(G, H, np.full(H.shape, 2.0)), vel, dt,
                                         np.zeros(H.shape))
    np.testing.assert_allclose(fdiv[1:], U * a / G.dx, rtol=1e-12)
    np.testing.assert_allclose(Hn[1:], H[1:] - dt * U * a / G.dx, rtol=1e-12)


def test_the_step_conserves_mass_up_to_its_accounted_fluxes():
    """periodic flux form: the divergence sums to zero over the grid, so the mass change
    equals the surface, basal and non-negativity totals"""
    G = grid()
    rng = np.random.default_rng(3)
    H = rng.uniform(0.0, 800.0, (G.Mx, G.My))
    mask = rng.choice([0.0, 2.0, 3.0, 4.0], size=H.shape)
    vel = rng.normal(0.0, 2e-5, (G.Mx, G.My, 2))
    cmb = rng.normal(0.0, 1e-5, H.shape)
    bmr = rng.uniform(0.0, 2e-8, H.shape)
    cfg = O.Config()
    dt = 3e6
    Hn, fdiv, tot = O.mass_continuity_step(G, cfg, inputs(G, H, mask), vel, dt, cmb, bmr)
    kg = cfg.ice_density * G.dx * G.dy
    change = float(np.sum(Hn - H)) * kg
    accounted = (tot["surface_ice_flux"] + tot["grounded_basal_ice_flux"] + tot["sub_shelf_ice_flux"]
                 + tot["sum_divQ_SSA"] + tot["nonneg_rule_flux"])
    assert change == pytest.approx(accounted, rel=1e-10)
    assert abs(tot["sum_divQ_SSA"]) <= 1e-9 * np.sum(np.abs(fdiv)) * dt * kg
    assert np.all(Hn >= 0.0)
    # no mass balance on ice-free ocean cells
    ocean = O.as_int(mask) == 4
    np.testing.assert_allclose(Hn[ocean], (H - dt * fdiv)[ocean].clip(min=0.0), rtol=1e-12, atol=1e-9)
