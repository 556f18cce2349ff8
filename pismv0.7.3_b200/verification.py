"""Verification test cases I, J and V for the SSA solve, and their exact solutions.

Host-side restatement of the reference's standalone SSA test drivers:

* test I  — src/base/stressbalance/ssa/tests/ssa_testi.cc:62-154 (Schoof plastic-till
  ice stream), exact solution src/verif/tests/exactTestsIJ.c:29-77;
* test J  — src/base/stressbalance/ssa/tests/ssa_testj.cc:64-134 (periodic linear
  ice shelf), exact solution src/verif/tests/exactTestsIJ.c:80-120;
* test V  — src/base/stressbalance/ssa/tests/ssa_test_cfbc.cc:44-180 (van der Veen
  shelf with the calving-front boundary condition);
* the error report of SSATestCase::report, SSATestCase.cc:173-253.

Each builder returns ``(grid, config, fields)`` where ``fields`` is a dict of
FP64 arrays indexed ``[i, j]`` (j contiguous; vectors ``[..., 2]`` interleaved)
that the solver consumes unchanged.
"""
from __future__ import annotations

import math

import numpy as np

from .config import SSAConfig, GridDesc, SECPERA, X_PERIODIC, Y_PERIODIC, XY_PERIODIC

MASK_ICE_FREE_BEDROCK = 0
MASK_GROUNDED = 2
MASK_FLOATING = 3
MASK_ICE_FREE_OCEAN = 4

_PI_EXACT = 3.14159265358979        # exactTestsIJ.c:27 (the file's own pi)
_SECPERA_EXACT = 31556926.0         # exactTestsIJ.c:28


# ---------------------------------------------------------------------------
# exact solutions
# ---------------------------------------------------------------------------
def exact_i(m: float, x, y):
    """Schoof's plastic-till stream (exactTestsIJ.c:29-77). Returns (bed, tauc, u, v)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    L = 40e3
    aspect = 0.05
    h0 = aspect * L
    theta = math.atan(0.001)
    rho, g = 910.0, 9.81
    f = rho * g * h0 * math.tan(theta)
    W = (m + 1.0) ** (1.0 / m) * L
    B = 3.7e8
    s = np.abs(y / L)
    tauc = f * np.power(s, m)
    bed = -x * math.tan(theta)
    C0 = 2.0 * (f / (B * h0)) ** 3.0 * L ** 4.0
    C1 = (m + 1.0) ** (4.0 / m)
    C2 = (m + 1.0) * C1
    C3 = (m + 1.0) * C2
    C4 = (m + 1.0) * C3
    z1 = (np.power(s, 4.0) - C1) / 4.0
    z2 = (np.power(s, m + 4.0) - C2) / ((m + 1.0) * (m + 4.0))
    z3 = (np.power(s, 2.0 * m + 4.0) - C3) / ((m + 1.0) * (m + 1.0) * (2.0 * m + 4.0))
    z4 = (np.power(s, 3.0 * m + 4.0) - C4) / ((m + 1.0) ** 3.0 * (3.0 * m + 4.0))
    u = np.where(np.abs(y) < W, -C0 * (z1 - 3.0 * z2 + 3.0 * z3 - z4), 0.0)
    v = np.zeros_like(u)
    return bed, tauc, u, v


_GAMMA_J = ((1.0854, 0.108, 0.0027),
            (0.402, 0.04, 0.001),
            (0.0402, 0.004, 0.0001))


def exact_j(x, y):
    """Periodic linearised ice shelf (exactTestsIJ.c:80-120). Returns (H, nu, u, v)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    pi = _PI_EXACT
    L = 300.0e3
    H0 = 500.0
    nu0 = 30.0 * 1.0e6 * _SECPERA_EXACT
    rho_ice, rho_sw, g = 910.0, 1028.0, 9.81
    C = rho_ice * g * (1.0 - rho_ice / rho_sw) * H0 / (2.0 * nu0)
    A = L / (4.0 * pi)
    H = H0 * (1.0 + 0.4 * np.cos(pi * x / L)) * (1.0 + 0.1 * np.cos(pi * y / L))
    nu = (nu0 * H0) / H
    uu = np.zeros(np.broadcast(x, y).shape)
    vv = np.zeros_like(uu)
    for k in range(-2, 3):
        for l in range(-2, 3):
            if k != 0 or l != 0:
                denom = float(k * k + l * l)
                kx = float(k) * pi * x / L
                ly = float(l) * pi * y / L
                trig = np.cos(kx) * np.sin(ly) + np.sin(kx) * np.cos(ly)
                Bc = (A / denom) * (C * _GAMMA_J[abs(k)][abs(l)]) * trig
                uu = uu + Bc * float(k)
                vv = vv + Bc * float(l)
    return H, nu, uu, vv


def van_der_veen_thickness(V0, H0, C, x):
    """ssa_test_cfbc.cc:44-48."""
    Q0 = V0 * H0
    return np.power(4 * C / Q0 * x + 1 / H0 ** 4, -0.25)


def van_der_veen_velocity(V0, H0, C, x):
    """ssa_test_cfbc.cc:51-54."""
    Q0 = V0 * H0
    return Q0 / van_der_veen_thickness(V0, H0, C, x)


# ---------------------------------------------------------------------------
# builders
# ---------------------------------------------------------------------------
def _empty_fields(Mx, My):
    return {
        "thickness": np.zeros((Mx, My)),
        "surface": np.zeros((Mx, My)),
        "bed": np.zeros((Mx, My)),
        "mask": np.full((Mx, My), float(MASK_GROUNDED)),   # SSATestCase.cc:110
        "tauc": np.zeros((Mx, My)),
        "bc_mask": np.zeros((Mx, My)),
        "bc_values": np.zeros((Mx, My, 2)),
        "melange": np.zeros((Mx, My)),                       # SSATestCase.cc:127
    }


def build_test_i(My: int = 61, Mx: int = 5, cfg: SSAConfig | None = None):
    """SSATestCaseI (ssa_testi.cc:71-145)."""
    m_schoof = 10.0
    L_schoof = 40e3
    H0 = 0.05 * L_schoof
    B_schoof = 3.7e8
    Ly = 3 * L_schoof
    Lx = max(60.0e3, ((Mx - 1) // 2) * (2.0 * Ly / (My - 1)))
    grid = GridDesc.shallow(Mx, My, Lx, Ly, periodicity=0)
    cfg = (cfg or SSAConfig()).copy()
    cfg.do_pseudo_plastic_till = False
    cfg.flow_law = "isothermal_glen"
    cfg.ice_softness = B_schoof ** (-cfg.ssa_Glen_exponent)
    cfg.compute_surf_grad_inward_ssa = True
    cfg.epsilon_ssa = 0.0
    f = _empty_fields(Mx, My)
    x, y = grid.x_coords(), grid.y_coords()
    X, Y = np.meshgrid(x, y, indexing="ij")
    f["thickness"][:] = H0
    theta = math.atan(0.001)
    fcoef = cfg.ice_density * cfg.standard_gravity * H0 * math.tan(theta)
    f["tauc"] = fcoef * np.power(np.abs(Y / L_schoof), m_schoof)
    bed, _, u, v = exact_i(m_schoof, X, Y)
    f["bed"] = bed
    f["surface"] = bed + H0
    I, J = np.meshgrid(np.arange(Mx), np.arange(My), indexing="ij")
    edge = (J == 0) | (J == My - 1) | (I == 0) | (I == Mx - 1)
    f["bc_mask"] = edge.astype(np.float64)
    f["bc_values"][..., 0] = np.where(edge, u, 0.0)
    f["bc_values"][..., 1] = np.where(edge, v, 0.0)
    return grid, cfg, f


def exact_velocity_i(grid: GridDesc):
    X, Y = np.meshgrid(grid.x_coords(), grid.y_coords(), indexing="ij")
    _, _, u, v = exact_i(10.0, X, Y)
    return np.stack([u, v], axis=-1)


def build_test_j(Mx: int = 61, My: int = 61, cfg: SSAConfig | None = None):
    """SSATestCaseJ (ssa_testj.cc:64-134)."""
    half = 300.0e3
    grid = GridDesc.shallow(Mx, My, half, half, periodicity=XY_PERIODIC)
    cfg = (cfg or SSAConfig()).copy()
    cfg.do_pseudo_plastic_till = False
    cfg.flow_law = "isothermal_glen"
    f = _empty_fields(Mx, My)
    f["tauc"][:] = 0.0
    f["bed"][:] = 0.0
    f["mask"][:] = MASK_FLOATING
    nu0 = 30.0 * 1.0e6 * SECPERA       # units::convert(30 MPa year -> Pa s)
    H0 = 500.0
    # strength extension forced above the thickest ice (ssa_testj.cc:98-99):
    # set_notional_strength(nu0*H0) then set_min_thickness(800) keeps nu*H = nu0*H0
    # (SSA.cc:41-58: each setter divides by the current minimum thickness)
    nu_c = (nu0 * H0) / cfg.min_thickness_strength_extension_ssa
    nuH_c = nu_c * cfg.min_thickness_strength_extension_ssa
    cfg.min_thickness_strength_extension_ssa = 800.0
    cfg.constant_nu_strength_extension_ssa = nuH_c / 800.0
    X, Y = np.meshgrid(grid.x_coords(), grid.y_coords(), indexing="ij")
    H, _, u, v = exact_j(X, Y)
    f["thickness"] = H
    f["surface"] = (1.0 - cfg.ice_density / cfg.sea_water_density) * H
    ic, jc = Mx // 2, My // 2
    f["bc_mask"][ic, jc] = 1.0
    f["bc_values"][ic, jc, 0] = u[ic, jc]
    f["bc_values"][ic, jc, 1] = v[ic, jc]
    return grid, cfg, f


def exact_velocity_j(grid: GridDesc):
    X, Y = np.meshgrid(grid.x_coords(), grid.y_coords(), indexing="ij")
    _, _, u, v = exact_j(X, Y)
    return np.stack([u, v], axis=-1)


_V0_V = 300.0 / SECPERA
_H0_V = 600.0
_C_V = 2.45e-18


def build_test_v(Mx: int = 201, My: int = 3, cfg: SSAConfig | None = None):
    """SSATestCaseCFBC (ssa_test_cfbc.cc:92-170)."""
    half = 250.0e3
    grid = GridDesc.shallow(Mx, My, half, half, periodicity=Y_PERIODIC)
    cfg = (cfg or SSAConfig()).copy()
    cfg.ice_softness = 1.9e8 ** (-cfg.ssa_Glen_exponent)
    cfg.compute_surf_grad_inward_ssa = False
    cfg.calving_front_stress_boundary_condition = True
    cfg.flow_law = "isothermal_glen"
    f = _empty_fields(Mx, My)
    f["tauc"][:] = 0.0
    f["bed"][:] = -1000.0
    x = grid.x_coords()
    Hx = van_der_veen_thickness(_V0_V, _H0_V, _C_V, x + grid.Lx)
    Hx[Mx - 1] = 0.0
    f["thickness"] = np.repeat(Hx[:, None], My, axis=1)
    f["mask"][:] = MASK_FLOATING
    f["mask"][Mx - 1, :] = MASK_ICE_FREE_OCEAN
    f["surface"] = (1.0 - cfg.ice_density / cfg.sea_water_density) * f["thickness"]
    f["bc_mask"][0, :] = 1.0
    f["bc_values"][0, :, 0] = _V0_V
    return grid, cfg, f


def exact_velocity_v(grid: GridDesc):
    x = grid.x_coords()
    u = van_der_veen_velocity(_V0_V, _H0_V, _C_V, x + grid.Lx)
    u[grid.Mx - 1] = 0.0
    out = np.zeros((grid.Mx, grid.My, 2))
    out[..., 0] = u[:, None]
    return out


_LIN = {"L": 50.0e3, "H0": 500.0, "nu0": 30.0 * 1.0e6 * SECPERA, "tauc0": 1.0e4, "v0": 100.0 / SECPERA}


def build_test_linear(Mx: int = 61, My: int = 61, cfg: SSAConfig | None = None):
    """SSATestCaseExp (ssa_test_linear.cc:52-118): flat 500 m slab, linearly viscous till
    (pseudo-plastic, q = 1), nu H fixed at nu0 H0 by the strength extension, exact
    u = v0 exp(-alpha (x - L)) prescribed on the edges."""
    L, H0, nu0, tauc0 = _LIN["L"], _LIN["H0"], _LIN["nu0"], _LIN["tauc0"]
    grid = GridDesc.shallow(Mx, My, L, L, periodicity=0)
    cfg = (cfg or SSAConfig()).copy()
    cfg.do_pseudo_plastic_till = True
    cfg.pseudo_plastic_q = 1.0
    # the strength extension covers every thickness, so the hardness never enters: the
    # isothermal law stands for the test case's flow law on its all-zero enthalpy
    cfg.flow_law = "isothermal_glen"
    # set_notional_strength(nu0 H0), then set_min_thickness(4000 * 10), which keeps nu H
    cfg.min_thickness_strength_extension_ssa = 4000.0 * 10
    cfg.constant_nu_strength_extension_ssa = nu0 * H0 / cfg.min_thickness_strength_extension_ssa
    cfg.compute_surf_grad_inward_ssa = True
    f = _empty_fields(Mx, My)
    f["thickness"][:] = H0
    f["surface"][:] = H0
    f["tauc"][:] = tauc0
    exact = exact_velocity_linear(grid, cfg)
    I, J = np.meshgrid(np.arange(Mx), np.arange(My), indexing="ij")
    edge = (J == 0) | (J == My - 1) | (I == 0) | (I == Mx - 1)
    f["bc_mask"] = edge.astype(np.float64)
    f["bc_values"] = np.where(edge[..., None], exact, 0.0)
    return grid, cfg, f


def exact_velocity_linear(grid: GridDesc, cfg: SSAConfig):
    """SSATestCaseExp::exactSolution, ssa_test_linear.cc:120-130."""
    alpha = math.sqrt((_LIN["tauc0"] / cfg.pseudo_plastic_uthreshold) / (4 * _LIN["nu0"] * _LIN["H0"]))
    X, _ = np.meshgrid(grid.x_coords(), grid.y_coords(), indexing="ij")
    out = np.zeros((grid.Mx, grid.My, 2))
    out[..., 0] = _LIN["v0"] * np.exp(-alpha * (X - _LIN["L"]))
    return out


_PLUG = {"H0": 2000.0, "L": 50.0e3, "dhdx": 0.001, "B0": 3.7e8}


def build_test_plug(Mx: int = 11, My: int = 61, glen_n: float = 3.0, cfg: SSAConfig | None = None):
    """SSATestCasePlug (ssa_test_plug.cc:55-158): a 2000 m slab on a uniform slope, no basal
    resistance, Dirichlet edges from the exact plug-flow speed."""
    H0, L, dhdx, B0 = _PLUG["H0"], _PLUG["L"], _PLUG["dhdx"], _PLUG["B0"]
    grid = GridDesc.shallow(Mx, My, L, L, periodicity=0)
    cfg = (cfg or SSAConfig()).copy()
    cfg.flow_law = "isothermal_glen"
    cfg.ice_softness = B0 ** (-glen_n)
    cfg.compute_surf_grad_inward_ssa = True
    cfg.epsilon_ssa = 0.0
    nuH = cfg.constant_nu_strength_extension_ssa * cfg.min_thickness_strength_extension_ssa
    cfg.min_thickness_strength_extension_ssa = H0 / 2   # set_min_thickness keeps nu H
    cfg.constant_nu_strength_extension_ssa = nuH / cfg.min_thickness_strength_extension_ssa
    f = _empty_fields(Mx, My)
    X, _ = np.meshgrid(grid.x_coords(), grid.y_coords(), indexing="ij")
    f["thickness"][:] = H0
    f["bed"] = -X * dhdx
    f["surface"] = f["bed"] + H0
    exact = exact_velocity_plug(grid, cfg)
    I, J = np.meshgrid(np.arange(Mx), np.arange(My), indexing="ij")
    edge = (J == 0) | (J == My - 1) | (I == 0) | (I == Mx - 1)
    f["bc_mask"] = edge.astype(np.float64)
    f["bc_values"] = np.where(edge[..., None], exact, 0.0)
    return grid, cfg, f


def exact_velocity_plug(grid: GridDesc, cfg: SSAConfig):
    """SSATestCasePlug::exactSolution, ssa_test_plug.cc:160-168 (the cube is Glen's n = 3)."""
    f = cfg.ice_density * cfg.standard_gravity * _PLUG["H0"] * _PLUG["dhdx"]
    _, Y = np.meshgrid(grid.x_coords(), grid.y_coords(), indexing="ij")
    out = np.zeros((grid.Mx, grid.My, 2))
    out[..., 0] = 0.5 * f ** 3 * _PLUG["L"] ** 4 / (_PLUG["B0"] * _PLUG["H0"]) ** 3 * (1 - (Y / _PLUG["L"]) ** 4)
    return out


def report(velocity: np.ndarray, exact: np.ndarray) -> dict:
    """SSATestCase::report (SSATestCase.cc:173-253): error norms in m/year and percent."""
    uerr = np.abs(velocity[..., 0] - exact[..., 0])
    verr = np.abs(velocity[..., 1] - exact[..., 1])
    N = uerr.size
    vecerr = np.sqrt(uerr * uerr + verr * verr)
    exactvelmax = float(np.max(np.sqrt(exact[..., 0] ** 2 + exact[..., 1] ** 2)))
    return {
        "maxvector": float(vecerr.max()) * SECPERA,
        "prcntavvec": float(vecerr.sum() / N) / exactvelmax * 100.0,
        "maxu": float(uerr.max()) * SECPERA,
        "maxv": float(verr.max()) * SECPERA,
        "avu": float(uerr.sum() / N) * SECPERA,
        "avv": float(verr.sum() / N) * SECPERA,
    }
