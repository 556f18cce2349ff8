"""The oracle's restatement of the consumers of the SSA velocity (ConstantInColumn, the
vertical velocity, the volumetric strain heating; PISMStressBalance.cc, SSB_Modifier.cc)
against closed-form answers: the reference's tests hold no vectors for these, so they are
pinned by fields whose differences and integrals are exact."""
import numpy as np
import pytest

from oracle import ssafd_oracle as O


def grid(Mx=9, My=7, Mz=6, Lz=3000.0):
    z = np.linspace(0.0, Lz, Mz)
    return O.Grid(Mx, My, 0.5 * (Mx - 1) * 5e3, 0.5 * (My - 1) * 4e3, z=z)


def inputs(G, mask, H=1000.0, E=None):
    shape = (G.Mx, G.My)
    return O.Inputs(thickness=np.full(shape, H) if np.isscalar(H) else H, surface=np.zeros(shape),
                    bed=np.zeros(shape), mask=mask, tauc=np.zeros(shape), enthalpy=E)


def linear_velocity(G, a, b):
    i, j = np.meshgrid(np.arange(G.Mx), np.arange(G.My), indexing="ij")
    return np.stack([a * i * G.dx, b * j * G.dy], axis=-1)


def test_constant_in_column_repeats_the_velocity():
    G = grid()
    vel = np.random.default_rng(0).normal(size=(G.Mx, G.My, 2))
    u3, v3 = O.constant_in_column(vel, len(G.z))
    for k in range(len(G.z)):
        np.testing.assert_array_equal(u3[..., k], vel[..., 0])
        np.testing.assert_array_equal(v3[..., k], vel[..., 1])


@pytest.mark.parametrize("bmr", [None, 3e-9])
def test_vertical_velocity_of_a_uniform_divergence(bmr):
    """u = a x, v = b y on icy cells: centred differences are exact, so away from the
    periodic seam w(z) = -bmr - (a + b) z"""
    G = grid()
    a, b = 2e-11, -5e-12
    vel = linear_velocity(G, a, b)
    u3, v3 = O.constant_in_column(vel, len(G.z))
    inp = inputs(G, np.full((G.Mx, G.My), 2.0))
    melt = None if bmr is None else np.full((G.Mx, G.My), bmr)
    w = O.vertical_velocity(G, inp, u3, v3, melt)
    expect = -(bmr or 0.0) - (a + b) * G.z
    np.testing.assert_allclose(w[1:-1, 1:-1], np.broadcast_to(expect, w[1:-1, 1:-1].shape), rtol=1e-12,
                               atol=1e-24)


def test_vertical_velocity_takes_one_sided_differences_at_margins():
    """an icy cell with an ice-free east neighbour uses (u_ij - u_w) / dx; an ice-free cell
    between two ice-free cells keeps the centred difference"""
    G = grid()
    mask = np.full((G.Mx, G.My), 2.0)
    mask[5, :] = 4.0   # ice-free ocean column i = 5
    mask[6, :] = 4.0
    rng = np.random.default_rng(1)
    vel = rng.normal(size=(G.Mx, G.My, 2)) * 1e-5
    u3, v3 = O.constant_in_column(vel, len(G.z))
    w = O.vertical_velocity(G, inputs(G, mask), u3, v3)
    u, v = vel[..., 0], vel[..., 1]
    i, j = 4, 3   # icy, ice-free to the east
    u_x = (u[i, j] - u[i - 1, j]) / G.dx
    v_y = (v[i, j + 1] - v[i, j - 1]) / (2 * G.dy)
    assert w[i, j, 1] == pytest.approx(-(u_x + v_y) * G.z[1], rel=1e-12)
    i = 5   # ice-free, icy to the west: one-sided towards the ice-free east
    u_x = (u[i + 1, j] - u[i, j]) / G.dx
    assert w[i, j, 1] == pytest.approx(-(u_x + (v[i, j + 1] - v[i, j - 1]) / (2 * G.dy)) * G.z[1], rel=1e-12)


def test_k_below_height_is_gsl_bisection():
    z = np.array([0.0, 10.0, 20.0, 40.0, 80.0])
    for h, k in [(0.0, 0), (5.0, 0), (10.0, 1), (39.9, 2), (40.0, 3), (79.0, 3), (80.0, 3)]:
        assert O.k_below_height(z, h) == k


def test_strain_heating_of_a_uniform_strain_rate():
    """isothermal Glen ice under a uniform strain rate: Sigma = 2 e^(-1/n) B D2^((1/n + 1) / 2)
    at levels up to kBelowHeight(H) and zero above, D2 = ((a + b)^2 + a^2 + b^2) / 2"""
    G = grid(Mz=8, Lz=3500.0)
    cfg = O.Config(flow_law="isothermal_glen", ice_softness=3.2e-24, ssa_enhancement_factor=2.0)
    a, b = 3e-11, 1e-11
    vel = linear_velocity(G, a, b)
    u3, v3 = O.constant_in_column(vel, len(G.z))
    H = np.full((G.Mx, G.My), 1600.0)
    sigma = O.volumetric_strain_heating(G, cfg, inputs(G, np.full((G.Mx, G.My), 2.0), H=H), u3, v3)
    n = cfg.ssa_Glen_exponent
    B = cfg.ice_softness ** (-1.0 / n)
    D2 = 0.5 * ((a + b) ** 2 + a * a + b * b)
    expect = 2.0 * cfg.ssa_enhancement_factor ** (-1.0 / n) * B * D2 ** (0.5 * (1.0 / n + 1.0))
    ks = O.k_below_height(G.z, 1600.0)   # z = 0, 500, 1000, 1500, 2000, ...: ks = 3
    assert ks == 3
    inner = sigma[1:-1, 1:-1]
    np.testing.assert_allclose(inner[..., :ks + 1], expect, rtol=1e-12)
    assert np.all(inner[..., ks + 1:] == 0.0)


def test_strain_heating_follows_the_enthalpy_dependent_hardness():
    """Paterson-Budd-type ice: each level's Sigma scales with that level's B(E, p)"""
    G = grid(Mz=6, Lz=2500.0)
    cfg = O.Config(flow_law="gpbld")
    vel = linear_velocity(G, 2e-11, 2e-11)
    u3, v3 = O.constant_in_column(vel, len(G.z))
    H = np.full((G.Mx, G.My), 2400.0)
    T = np.linspace(250.0, 268.0, len(G.z))
    E = np.empty((G.Mx, G.My, len(G.z)))
    for k in range(len(G.z)):
        E[..., k] = O.ec_enthalpy(cfg, T[k], 0.0, O.ec_pressure(cfg, 2400.0 - G.z[k]))
    sigma = O.volumetric_strain_heating(G, cfg, inputs(G, np.full((G.Mx, G.My), 2.0), H=H, E=E), u3, v3)
    B = np.array([O.hardness_parameter(cfg, E[4, 3, k], O.ec_pressure(cfg, 2400.0 - G.z[k]))
                  for k in range(len(G.z))])
    ks = O.k_below_height(G.z, 2400.0)
    ratio = sigma[4, 3, :ks + 1] / B[:ks + 1]
    np.testing.assert_allclose(ratio, ratio[0], rtol=1e-12)
