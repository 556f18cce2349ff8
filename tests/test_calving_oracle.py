"""The oracle's restatement of the strain-rate / eigen-calving path (ShallowStressBalance.cc:224-386,
PISMEigenCalving.cc:77-493) against closed-form answers: the reference's tests print no vectors
for it, so it is pinned by velocity fields whose derivatives are exact and by mask patterns
whose outcome follows from the reference's (i, j) loop order."""
import numpy as np
import pytest

from oracle import ssafd_oracle as O

F, G_, OC, B = O.MASK_FLOATING, O.MASK_GROUNDED, O.MASK_ICE_FREE_OCEAN, O.MASK_ICE_FREE_BEDROCK


def grid(Mx=16, My=14, d=5e3):
    return O.Grid(Mx, My, 0.5 * (Mx - 1) * d, 0.5 * (My - 1) * d)


def linear_velocity(G, a, b, c, d):
    x = np.arange(G.Mx)[:, None] * G.dx * np.ones((1, G.My))
    y = np.arange(G.My)[None, :] * G.dy * np.ones((G.Mx, 1))
    return np.stack([a * x + b * y, c * x + d * y], axis=-1)


def test_principal_strain_rates_of_a_linear_field():
    G = grid()
    a, b, c, d = 1e-9, 2e-9, -3e-9, 4e-9
    e = O.principal_strain_rates(G, np.full((G.Mx, G.My), 2.0), linear_velocity(G, a, b, c, d))
    ev = np.linalg.eigvalsh(np.array([[a, 0.5 * (b + c)], [0.5 * (b + c), d]]))[::-1]
    np.testing.assert_allclose(e[1:-1, 1:-1], np.broadcast_to(ev, e[1:-1, 1:-1].shape), rtol=1e-6)
    assert np.all(e[..., 0] >= e[..., 1])


def test_one_sided_differences_next_to_ice_free_cells():
    G = grid()
    rng = np.random.default_rng(1)
    vel = rng.normal(size=(G.Mx, G.My, 2))
    M = np.full((G.Mx, G.My), 2.0)
    M[6, 5] = 4.0   # ice-free east of (5, 5)
    M[5, 4] = 0.0   # ice-free south of (5, 5)
    M[9, 5] = M[11, 5] = 4.0   # (10, 5): both x neighbours ice-free
    ux, uy, vx, vy = O._velocity_gradient(G, O.as_int(M), vel)
    u, v = vel[..., 0], vel[..., 1]
    assert ux[5, 5] == (u[5, 5] - u[4, 5]) / G.dx
    assert uy[5, 5] == (u[5, 6] - u[5, 5]) / G.dy
    assert ux[10, 5] == 0.0 and vx[10, 5] == 0.0
    e = O.principal_strain_rates(G, M, vel)
    assert np.all(e[6, 5] == 0.0) and np.all(e[5, 4] == 0.0)


def test_stresses_follow_the_effective_viscosity():
    G = grid()
    cfg = O.Config()
    a, b, c, d = 2e-10, 1e-10, 3e-10, -1e-10
    s = O.deviatoric_stresses_2d(G, cfg, np.full((G.Mx, G.My), 3.0), linear_velocity(G, a, b, c, d))
    n = cfg.ssa_Glen_exponent
    hardness = cfg.ice_softness ** (-1.0 / n)
    gamma = 0.5 * (a * a + d * d + (a + d) ** 2 + 0.5 * (b + c) ** 2)
    nu = 0.5 * hardness * (O.schoof_reg(cfg) + gamma) ** ((1.0 - n) / (2.0 * n))
    np.testing.assert_allclose(s[7, 7], [nu * a, nu * d, 0.5 * nu * (b + c)], rtol=1e-6)


def tongue_mask(Mx=16, My=14):
    """a floating block at i <= 2 with a one-cell tongue pointing east along j = 6 (i = 3..5),
    and a floating block at i >= 12 with one pointing west (i = 8..10); ocean elsewhere"""
    M = np.full((Mx, My), OC)
    M[:3, :] = F
    M[3:6, 6] = F
    M[12:, :] = F
    M[8:11, 6] = F
    return M


def test_remove_narrow_tongues_follows_the_loop_order():
    """the east tongue loses its tip only (its other cells were visited before the tip went);
    the west tongue's tip goes first, so the next cell, visited later, sees it gone and
    goes too, and so on up to the cell next to the block"""
    M = tongue_mask()
    H = np.where(M == F, 100.0, 0.0)
    Mn, Hn = O.remove_narrow_tongues(M, H)
    gone = (M != Mn)
    assert sorted(zip(*np.nonzero(gone))) == [(5, 6), (8, 6), (9, 6)]
    assert np.all(Mn[gone] == OC) and np.all(Hn[gone] == 0.0)
    np.testing.assert_array_equal(Hn[~gone], H[~gone])


def test_isolated_cells_and_grounded_tips():
    """a floating cell with no icy neighbour stays (no clause holds); of a grounded pair in
    ice-free ocean the west cell goes (visited first, its east neighbour still icy) and the
    east cell, now alone, stays; a grounded tip whose other side is ice-free bedrock stays"""
    M = np.full((10, 10), OC)
    M[5, 5] = F
    M[2:4, 2] = G_            # grounded pair in ice-free ocean
    M[7:9, 8] = G_            # grounded pair with bedrock north-east of it
    M[8:10, 9] = B
    Mn, _ = O.remove_narrow_tongues(M, np.ones(M.shape))
    assert Mn[5, 5] == F
    assert Mn[2, 2] == OC and Mn[3, 2] == G_
    assert Mn[7, 8] == G_ and Mn[8, 8] == G_


def spreading_shelf(K=1e17):
    """a floating shelf (i <= 9) spreading with u = a x, v = b y, ocean beyond"""
    G = grid(20, 16)
    M = np.full((G.Mx, G.My), OC)
    M[:10, :] = F
    H = np.where(M == F, 400.0, 0.0)
    a, b = 3e-10, 1e-10
    vel = linear_velocity(G, a, 0.0, 0.0, b)
    return G, M, H, vel, a, b, K


def test_eigen_calving_rate_at_the_front():
    """at the front cell (10, 7): the cells two away that are floating and not at the margin
    are (8, 7) only ((12, 7) is ocean; (10, 5), (10, 9) are ocean), so e1 = a, e2 = b and
    the calving rate is K a b H / dx with H the one floating neighbour's 400 m"""
    G, M, H, vel, a, b, K = spreading_shelf()
    dt = 1e5
    Href = np.zeros(M.shape)
    Href[10, :] = 50.0   # every front cell of the shelf keeps some Href: nothing is cut
    Mn, Hrefn, Hn = O.eigen_calving(G, M, Href, H, vel, dt, K)
    rate = K * a * b * 400.0 / G.dx
    assert Hrefn[10, 7] == pytest.approx(max(50.0 - rate * dt, 0.0), rel=1e-9)
    assert 50.0 - rate * dt > 0.0   # nothing cut: the mask and thickness stay
    np.testing.assert_array_equal(Mn, M)
    np.testing.assert_array_equal(Hn, H)


def test_eigen_calving_cuts_the_floating_neighbour():
    """Href goes negative: the loss goes to the one floating neighbour, which is cut"""
    G, M, H, vel, a, b, K = spreading_shelf(K=1e19)
    dt = 3e6
    Mn, Hrefn, Hn = O.eigen_calving(G, M, np.zeros(M.shape), H, vel, dt, K)
    rate = K * a * b * 400.0 / G.dx
    loss = rate * dt   # Href = 0 - rate dt < 0, shared by one neighbour
    assert Mn[9, 7] == OC and Hn[9, 7] == 0.0
    assert Hrefn[9, 7] == pytest.approx(max(400.0 - loss, 0.0), abs=1e-9)
    assert Hrefn[10, 7] == 0.0


def test_max_timestep():
    G, M, H, vel, a, b, K = spreading_shelf()
    dt, rmax, rmean, count = O.eigen_calving_max_timestep(G, M, vel, K)
    assert count > 0 and rmax == pytest.approx(K * a * b, rel=1e-6)
    assert rmean <= rmax
    eps = 0.001 / (G.dx + G.dy) / O.SECPERA
    assert dt == pytest.approx(max(1.0 / (rmax / G.dx + eps), 0.001 * O.SECPERA))
    # no spreading, no calving: the time step is bounded by epsilon alone
    dt0, r0, m0, c0 = O.eigen_calving_max_timestep(G, M, np.zeros_like(vel), K)
    assert (r0, m0, c0) == (0.0, 0.0, 0.0) and dt0 == pytest.approx(1.0 / eps)
