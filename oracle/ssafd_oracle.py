"""CPU oracle for the PISM v0.7.3 SSAFD solve — TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
The GPU solver in ``pismv0.7.3_b200`` never routes through it.

It restates, in vectorised numpy (FP64, no FMA contraction), the arithmetic of
the reference's finite-difference shallow-shelf solver.  Every function names
the reference file:line it follows (paths relative to the PISM source tree):

* driving stress            src/base/stressbalance/ssa/SSA.cc:211-353
* right-hand side           src/base/stressbalance/ssa/SSAFD.cc:282-417
* matrix assembly           src/base/stressbalance/ssa/SSAFD.cc:496-811
* staggered hardness        src/base/stressbalance/ssa/SSAFD.cc:1192-1246
* fracture softening        src/base/stressbalance/ssa/SSAFD.cc:1282-1310
* nu*H (plain / CFBC)       src/base/stressbalance/ssa/SSAFD.cc:1359-1421 / 1441-1582
* nu*H norm                 src/base/stressbalance/ssa/SSAFD.cc:1170-1189
* Picard loop + strategies  src/base/stressbalance/ssa/SSAFD.cc:869-1155
* flow laws                 src/base/rheology/flowlaws.{hh,cc}
* basal resistance          src/base/basalstrength/basal_resistance.cc:46-50,154-163
* mask predicates           src/base/util/Mask.hh:28-65
* enthalpy converter        src/base/enthalpyConverter.cc:92-290

Grid conventions (src/base/util/IceGrid.cc:540-610, 800-823): arrays are indexed
``[i, j]`` (i = x, j = y, j contiguous), vectors interleave (u, v), staggered
fields store (east face, north face) per cell, and every neighbour access wraps
periodically because the PETSc DMDA is created periodic in both directions.

The linear solve of each Picard step is a direct sparse LU (scipy SuperLU) of
the exact 18-column-per-row matrix, i.e. the tight answer PETSc's KSP would
converge to.  Parity is pinned by ``tests/golden`` (verification tests I, J, V
of test/regression/ssa/*.sh, the flow-law tables of test/regression/test_2x.sh
and exactTestsIJ.c vectors produced by compiling the reference's own C file).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# UDUNITS-2 "year" (365.242198781 days); PISM converts m/year <-> m/s through it.
SECPERA = 31556925.9747

MASK_ICE_FREE_BEDROCK = 0
MASK_GROUNDED = 2
MASK_FLOATING = 3
MASK_ICE_FREE_OCEAN = 4

X_PERIODIC = 1
Y_PERIODIC = 2


# ---------------------------------------------------------------------------
# configuration (defaults from src/pism_config.cdl, converted to SI)
# ---------------------------------------------------------------------------
@dataclass
class Config:
    ice_density: float = 910.0                       # pism_config.cdl:993
    sea_water_density: float = 1028.0                # :1140
    standard_gravity: float = 9.81                   # :1188
    sea_level: float = 0.0                           # ShallowStressBalance.cc:41
    epsilon_ssa: float = 1.0e13                      # :353
    ssafd_relative_convergence: float = 1.0e-4       # :617
    max_iterations_ssafd: int = 300                  # :566
    ssafd_nuH_iter_failure_underrelaxation: float = 0.8  # :623
    min_thickness_strength_extension_ssa: float = 50.0    # :358
    constant_nu_strength_extension_ssa: float = 9.48680701906572e14  # :363
    plastic_regularization: float = 0.01 / SECPERA   # :599 (m/yr -> m/s)
    do_pseudo_plastic_till: bool = False             # :65
    pseudo_plastic_q: float = 0.25                   # :605
    pseudo_plastic_uthreshold: float = 100.0 / SECPERA  # :611
    sliding_scale_factor_reduces_tauc: float = -1.0  # :392
    beta_ice_free_bedrock: float = 1.8e9             # :397
    calving_front_stress_boundary_condition: bool = False  # :73
    ssa_dirichlet_bc: bool = False                   # :161
    sub_groundingline: bool = False                  # :197
    nu_bedrock_set: bool = False                     # :192
    nu_bedrock: float = 5.0e15                       # :188
    surface_gradient_method: str = "haseloff"        # :1272
    compute_surf_grad_inward_ssa: bool = False       # :156
    flow_law: str = "gpbld"                          # :1100 (ssa_flow_law)
    ssa_Glen_exponent: float = 3.0                   # :1015
    ssa_enhancement_factor: float = 1.0              # :287
    ice_softness: float = 3.1689e-24                 # :1020
    Schoof_regularizing_length: float = 1000.0e3     # :1050 (km -> m)
    Schoof_regularizing_velocity: float = 1.0 / SECPERA  # :1055 (m/yr -> m/s)
    Paterson_Budd_A_cold: float = 3.61e-13           # :1060
    Paterson_Budd_A_warm: float = 1.73e3             # :1065
    Paterson_Budd_Q_cold: float = 6.0e4              # :1070
    Paterson_Budd_Q_warm: float = 13.9e4             # :1075
    Paterson_Budd_critical_temperature: float = 263.15  # :1080
    ideal_gas_constant: float = 8.31441              # :1193
    gpbld_water_frac_coeff: float = 181.25           # :1115
    gpbld_water_frac_observed_limit: float = 0.01    # :1120
    Hooke_A: float = 4.42165e-9                      # :1025
    Hooke_Q: float = 7.88e4                          # :1030
    Hooke_C: float = 0.16612                         # :1035
    Hooke_k: float = 1.17                            # :1040
    Hooke_Tr: float = 273.39                         # :1045
    beta_CC: float = 7.9e-8                          # :963
    ice_specific_heat_capacity: float = 2009.0       # :1003
    water_latent_heat_fusion: float = 3.34e5         # :983
    surface_pressure: float = 0.0                    # :968
    water_melting_point_temperature: float = 273.15  # :973
    enthalpy_converter_reference_temperature: float = 223.15  # :978
    do_fracture_density: bool = False
    fracture_density_softening_lower_limit: float = 1.0  # :115
    brutal_sliding: bool = False                     # :292
    brutal_sliding_scale: float = 1.0                # :298
    mask_icefree_thickness_standard: float = 0.01    # :1225
    mask_is_floating_thickness_standard: float = 1.0 # :1230
    scaling: float = 1.0e9                           # SSAFD.cc:93 (m_scaling)

    def copy(self, **kw) -> "Config":
        return replace(self, **kw)


@dataclass
class Grid:
    """Horizontal grid, src/base/util/IceGrid.cc:540-610 (compute_horizontal_*)."""
    Mx: int
    My: int
    Lx: float
    Ly: float
    x0: float = 0.0
    y0: float = 0.0
    periodicity: int = 0
    z: np.ndarray | None = None  # vertical levels (enthalpy columns)

    @property
    def dx(self) -> float:
        if self.periodicity & X_PERIODIC:
            return 2.0 * self.Lx / self.Mx
        return 2.0 * self.Lx / (self.Mx - 1)

    @property
    def dy(self) -> float:
        if self.periodicity & Y_PERIODIC:
            return 2.0 * self.Ly / self.My
        return 2.0 * self.Ly / (self.My - 1)

    @staticmethod
    def _coords(M, delta, vmin, vmax, periodic):
        if periodic:
            r = vmin + (np.arange(M) + 0.5) * delta
            r[M - 1] = vmax - 0.5 * delta
        else:
            r = vmin + np.arange(M) * delta
            r[M - 1] = vmax
        return r

    @property
    def x(self) -> np.ndarray:
        return self._coords(self.Mx, self.dx, self.x0 - self.Lx, self.x0 + self.Lx,
                            bool(self.periodicity & X_PERIODIC))

    @property
    def y(self) -> np.ndarray:
        return self._coords(self.My, self.dy, self.y0 - self.Ly, self.y0 + self.Ly,
                            bool(self.periodicity & Y_PERIODIC))


# ---------------------------------------------------------------------------
# helpers: periodic neighbours and mask predicates
# ---------------------------------------------------------------------------
def nb(a: np.ndarray, di: int, dj: int) -> np.ndarray:
    """a(i+di, j+dj) with the DMDA's periodic wrap (IceGrid.cc:807-819)."""
    return np.roll(a, shift=(-di, -dj), axis=(0, 1))


def as_int(mask: np.ndarray) -> np.ndarray:
    """IceModelVec2Int::as_int, IceModelVec_inline.hh:94-100."""
    return np.floor(np.asarray(mask, dtype=np.float64) + 0.5).astype(np.int64)


# Mask.hh:28-65
def m_ocean(M):
    return M >= MASK_FLOATING


def m_grounded(M):
    return ~m_ocean(M)


def m_icy(M):
    return (M == MASK_GROUNDED) | (M == MASK_FLOATING)


def m_grounded_ice(M):
    return m_icy(M) & m_grounded(M)


def m_floating_ice(M):
    return m_icy(M) & m_ocean(M)


def m_ice_free(M):
    return ~m_icy(M)


def m_ice_free_ocean(M):
    return m_ocean(M) & m_ice_free(M)


def m_ice_free_land(M):
    return m_grounded(M) & m_ice_free(M)


def geometry_mask_surface(cfg: Config, bed, thickness):
    """GeometryCalculator::compute, Mask.hh:82-118 (dry simulation off)."""
    alpha = 1.0 - cfg.ice_density / cfg.sea_water_density
    hgrounded = bed + thickness
    hfloating = cfg.sea_level + alpha * thickness
    is_floating = hfloating > hgrounded + cfg.mask_is_floating_thickness_standard
    ice_free = thickness < cfg.mask_icefree_thickness_standard
    surface = np.where(is_floating, hfloating, hgrounded)
    mask = np.where(is_floating,
                    np.where(ice_free, MASK_ICE_FREE_OCEAN, MASK_FLOATING),
                    np.where(ice_free, MASK_ICE_FREE_BEDROCK, MASK_GROUNDED))
    return mask.astype(np.float64), surface


# ---------------------------------------------------------------------------
# enthalpy converter (enthalpyConverter.cc:56-290) and flow laws (flowlaws.*)
# ---------------------------------------------------------------------------
def ec_pressure(cfg: Config, depth):
    """EnthalpyConverter::pressure, enthalpyConverter.cc:92-98."""
    depth = np.asarray(depth, dtype=np.float64)
    return np.where(depth > 0.0,
                    cfg.surface_pressure + cfg.ice_density * cfg.standard_gravity * depth,
                    cfg.surface_pressure)


def ec_melting_temperature(cfg, P):
    return cfg.water_melting_point_temperature - cfg.beta_CC * P          # :140-142


def ec_enthalpy_cts(cfg, P):
    return cfg.ice_specific_heat_capacity * (ec_melting_temperature(cfg, P)
                                             - cfg.enthalpy_converter_reference_temperature)  # :152-154


def ec_temperature(cfg, E, P):
    """EnthalpyConverter::temperature_impl, enthalpyConverter.cc:184-199."""
    return np.where(E < ec_enthalpy_cts(cfg, P),
                    E / cfg.ice_specific_heat_capacity + cfg.enthalpy_converter_reference_temperature,
                    ec_melting_temperature(cfg, P))


def ec_pressure_adjusted_temperature(cfg, E, P):
    return ec_temperature(cfg, E, P) - ec_melting_temperature(cfg, P) + cfg.water_melting_point_temperature


def ec_water_fraction(cfg, E, P):
    """enthalpyConverter.cc:217-231."""
    Es = ec_enthalpy_cts(cfg, P)
    return np.where(E <= Es, 0.0, (E - Es) / cfg.water_latent_heat_fusion)


def ec_enthalpy(cfg, T, omega, P):
    """enthalpyConverter.cc:252-279 (checks omitted)."""
    Tm = ec_melting_temperature(cfg, P)
    return np.where(T < Tm, cfg.ice_specific_heat_capacity * (T - cfg.enthalpy_converter_reference_temperature),
                    ec_enthalpy_cts(cfg, P) + omega * cfg.water_latent_heat_fusion)


def softness_paterson_budd(cfg, T_pa):
    """FlowLaw::softness_parameter_paterson_budd, flowlaws.cc:90-95."""
    R = cfg.ideal_gas_constant
    return np.where(T_pa < cfg.Paterson_Budd_critical_temperature,
                    cfg.Paterson_Budd_A_cold * np.exp(-cfg.Paterson_Budd_Q_cold / (R * T_pa)),
                    cfg.Paterson_Budd_A_warm * np.exp(-cfg.Paterson_Budd_Q_warm / (R * T_pa)))


def softness(cfg: Config, E, P):
    """softness_parameter(E, p) of the ssa flow law (flowlaws.cc:209-253, flowlaws.hh:201-325)."""
    law = cfg.flow_law
    E = np.asarray(E, dtype=np.float64)
    P = np.asarray(P, dtype=np.float64)
    if law == "isothermal_glen":
        return np.full(np.broadcast(E, P).shape, cfg.ice_softness)
    R = cfg.ideal_gas_constant
    if law == "gpbld":
        Es = ec_enthalpy_cts(cfg, P)
        T_pa = ec_pressure_adjusted_temperature(cfg, E, P)
        omega = np.minimum(ec_water_fraction(cfg, E, P), cfg.gpbld_water_frac_observed_limit)
        cold = softness_paterson_budd(cfg, T_pa)
        warm = softness_paterson_budd(cfg, cfg.water_melting_point_temperature) * \
            (1.0 + cfg.gpbld_water_frac_coeff * omega)
        return np.where(E < Es, cold, warm)
    T_pa = ec_pressure_adjusted_temperature(cfg, E, P)
    if law == "pb":
        return softness_paterson_budd(cfg, T_pa)
    if law == "arr":
        return cfg.Paterson_Budd_A_cold * np.exp(-cfg.Paterson_Budd_Q_cold / (R * T_pa))
    if law == "arrwarm":
        return cfg.Paterson_Budd_A_warm * np.exp(-cfg.Paterson_Budd_Q_warm / (R * T_pa))
    if law == "hooke":
        return cfg.Hooke_A * np.exp(-cfg.Hooke_Q / (R * T_pa)
                                    + 3.0 * cfg.Hooke_C * np.power(cfg.Hooke_Tr - T_pa, -cfg.Hooke_k))
    raise ValueError(f"unknown flow law {law}")


def hardness_parameter(cfg: Config, E, P):
    """FlowLaw::hardness_parameter = softness^(-1/n), flowlaws.cc:104-106."""
    if cfg.flow_law == "isothermal_glen":
        return np.full(np.broadcast(np.asarray(E), np.asarray(P)).shape,
                       cfg.ice_softness ** (-1.0 / cfg.ssa_Glen_exponent))
    return np.power(softness(cfg, E, P), -1.0 / cfg.ssa_Glen_exponent)


def k_below_height(z: np.ndarray, height):
    """IceGrid::kBelowHeight via gsl_interp_accel_find: largest k in [0, Mz-2] with z[k] <= h."""
    k = np.searchsorted(z, height, side="right") - 1
    return np.clip(k, 0, len(z) - 2)


def averaged_hardness(cfg: Config, H, z, E_col):
    """FlowLaw::averaged_hardness, flowlaws.cc:141-185 (isothermal: flowlaws.hh:222-225).

    H: (n,) thicknesses, E_col: (n, Mz) enthalpy columns."""
    H = np.asarray(H, dtype=np.float64)
    if cfg.flow_law == "isothermal_glen":
        return np.full(H.shape, cfg.ice_softness ** (-1.0 / cfg.ssa_Glen_exponent))
    kb = k_below_height(z, H)
    B = np.zeros_like(H)
    h0 = hardness_parameter(cfg, E_col[:, 0], ec_pressure(cfg, H))
    for k in range(1, len(z)):
        active = k <= kb
        h1 = hardness_parameter(cfg, E_col[:, k], ec_pressure(cfg, H - z[k]))
        B = np.where(active, B + (z[k] - z[k - 1]) * (h0 + h1), B)
        h0 = np.where(active, h1, h0)
    B = B * 0.5
    depth = H - z[kb]
    B = B + depth * hardness_parameter(cfg, E_col[np.arange(len(H)), kb], ec_pressure(cfg, depth))
    return np.where(H > 0, B / np.where(H > 0, H, 1.0), 0.0)


def schoof_reg(cfg: Config) -> float:
    """FlowLaw::m_schoofReg, flowlaws.cc:83-85."""
    return (cfg.Schoof_regularizing_velocity / cfg.Schoof_regularizing_length) ** 2


def second_invariant_2d(u_x, u_y, v_x, v_y):
    """flowlaws.hh:36-39."""
    return 0.5 * (u_x * u_x + v_y * v_y + (u_x + v_y) * (u_x + v_y) + 0.5 * ((u_y + v_x) * (u_y + v_x)))


def effective_viscosity(cfg: Config, hardness, gamma):
    """FlowLaw::effective_viscosity, flowlaws.hh:100-112."""
    n = cfg.ssa_Glen_exponent
    return 0.5 * hardness * np.power(schoof_reg(cfg) + gamma, (1.0 - n) / (2.0 * n))


def basal_drag(cfg: Config, tauc, u, v):
    """IceBasalResistance{Plastic,PseudoPlastic}Law::drag, basal_resistance.cc:46-50,154-163."""
    magreg2 = cfg.plastic_regularization ** 2 + u * u + v * v
    if not cfg.do_pseudo_plastic_till:
        return tauc / np.sqrt(magreg2)
    q = cfg.pseudo_plastic_q
    if cfg.sliding_scale_factor_reduces_tauc > 0.0:
        Aq = cfg.sliding_scale_factor_reduces_tauc ** q
        return (tauc / Aq) * np.power(magreg2, 0.5 * (q - 1)) * cfg.pseudo_plastic_uthreshold ** (-q)
    return tauc * np.power(magreg2, 0.5 * (q - 1)) * cfg.pseudo_plastic_uthreshold ** (-q)


# ---------------------------------------------------------------------------
# SSA inputs
# ---------------------------------------------------------------------------
@dataclass
class Inputs:
    """Fields the SSA fetches in SSA::init_impl (SSA.cc:134-184), all (Mx, My) FP64."""
    thickness: np.ndarray
    surface: np.ndarray
    bed: np.ndarray
    mask: np.ndarray
    tauc: np.ndarray
    bc_mask: np.ndarray | None = None      # 1 = Dirichlet location
    bc_values: np.ndarray | None = None    # (Mx, My, 2), m/s
    melange: np.ndarray | None = None      # melange back pressure fraction
    gl_mask: np.ndarray | None = None      # sub-grid grounded fraction
    enthalpy: np.ndarray | None = None     # (Mx, My, Mz)
    fracture_density: np.ndarray | None = None


# ---------------------------------------------------------------------------
# driving stress and right-hand side
# ---------------------------------------------------------------------------
def driving_stress(grid: Grid, cfg: Config, inp: Inputs) -> np.ndarray:
    """SSA::compute_driving_stress, SSA.cc:211-353.  Returns (Mx, My, 2)."""
    H = inp.thickness
    s = inp.surface
    b = inp.bed
    M = as_int(inp.mask)
    n = cfg.ssa_Glen_exponent
    etapow = (2.0 * n + 2.0) / n
    invpow = 1.0 / etapow
    dinvpow = (-n - 2.0) / (2.0 * n + 2.0)
    minThickEtaTransform = 5.0
    dx, dy = grid.dx, grid.dy
    use_eta = cfg.surface_gradient_method == "eta"
    cfbc = cfg.calving_front_stress_boundary_condition

    pressure = ec_pressure(cfg, H)
    Mx, My = H.shape

    # eta branch (grounded and use_eta)
    with np.errstate(all="ignore"):
        myH = np.where(H < minThickEtaTransform, minThickEtaTransform, H)
        eta = np.power(myH, etapow)
        factor = invpow * np.power(eta, dinvpow)
        Hp = np.power(H, etapow)
        hx_eta = np.where(H > 0.0, factor * (nb(Hp, 1, 0) - nb(Hp, -1, 0)) / (2 * dx), 0.0)
        hy_eta = np.where(H > 0.0, factor * (nb(Hp, 0, 1) - nb(Hp, 0, -1)) / (2 * dy), 0.0)
    hx_eta = hx_eta + (nb(b, 1, 0) - nb(b, -1, 0)) / (2 * dx)   # IceModelVec2S::diff_x
    hy_eta = hy_eta + (nb(b, 0, 1) - nb(b, 0, -1)) / (2 * dy)

    if cfg.compute_surf_grad_inward_ssa:
        # IceModelVec2S::diff_x_p / diff_y_p, iceModelVec2.cc:501-530
        hx = (nb(s, 1, 0) - nb(s, -1, 0)) / (2 * dx)
        hy = (nb(s, 0, 1) - nb(s, 0, -1)) / (2 * dy)
        if not (grid.periodicity & X_PERIODIC):
            hx[0, :] = (s[1, :] - s[0, :]) / dx
            hx[Mx - 1, :] = (s[Mx - 1, :] - s[Mx - 2, :]) / dx
        if not (grid.periodicity & Y_PERIODIC):
            hy[:, 0] = (s[:, 1] - s[:, 0]) / dy
            hy[:, My - 1] = (s[:, My - 1] - s[:, My - 2]) / dy
    else:
        g = m_grounded(M)
        fl = m_floating_ice(M)
        ifo = m_ice_free_ocean(M)
        icy = m_icy(M)
        ifr = m_ice_free(M)

        def one_sided_weights(di, dj):
            Mn_g = nb(g, di, dj)
            Mn_fl = nb(fl, di, dj)
            Mn_ifo = nb(ifo, di, dj)
            w = np.ones(H.shape)
            zero = (g & Mn_fl) | (fl & Mn_g) | (fl & Mn_ifo)
            if cfbc:
                zero = zero | (icy & nb(ifr, di, dj))
            w[zero] = 0.0
            return w

        east = one_sided_weights(1, 0)
        west = one_sided_weights(-1, 0)
        north = one_sided_weights(0, 1)
        south = one_sided_weights(0, -1)
        dxE = (nb(s, 1, 0) - s) / dx          # diff_x_stagE(i, j)
        dxW = (s - nb(s, -1, 0)) / dx         # diff_x_stagE(i-1, j)
        dyN = (nb(s, 0, 1) - s) / dy          # diff_y_stagN(i, j)
        dyS = (s - nb(s, 0, -1)) / dy         # diff_y_stagN(i, j-1)
        with np.errstate(all="ignore"):
            hx = np.where(east + west > 0, 1.0 / (west + east) * (west * dxW + east * dxE), 0.0)
            hy = np.where(north + south > 0, 1.0 / (south + north) * (south * dyS + north * dyN), 0.0)

    if use_eta:
        gr = m_grounded(M)
        hx = np.where(gr, hx_eta, hx)
        hy = np.where(gr, hy_eta, hy)

    taud = np.zeros((Mx, My, 2))
    pos = pressure > 0.0
    taud[..., 0] = np.where(pos, -pressure * hx, 0.0)
    taud[..., 1] = np.where(pos, -pressure * hy, 0.0)
    return taud


def is_marginal(M, ssa_dirichlet_bc: bool):
    """SSAFD::is_marginal, SSAFD.cc:1657-1682."""
    pred = m_ice_free if ssa_dirichlet_bc else m_ice_free_ocean
    any_nb = np.zeros(M.shape, dtype=bool)
    for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (1, -1), (-1, 1), (-1, -1)):
        any_nb |= pred(nb(M, di, dj))
    return m_icy(M) & any_nb


def cfbc_weights(M, cfg: Config):
    """The 12 integer weights aMn..bMe of SSAFD.cc:594-684, as float arrays (all ones without CFBC)."""
    names = ["aMn", "aPn", "aMM", "aPP", "aMs", "aPs", "bPw", "bPP", "bPe", "bMw", "bMM", "bMe"]
    w = {k: np.ones(M.shape) for k in names}
    if not cfg.calving_front_stress_boundary_condition:
        return w
    bb = cfg.ssa_dirichlet_bc
    f = m_ice_free_ocean if bb else m_ice_free
    marg = is_marginal(M, bb)
    e, wv, n, s = f(nb(M, 1, 0)), f(nb(M, -1, 0)), f(nb(M, 0, 1)), f(nb(M, 0, -1))
    ne, se, nw, sw = f(nb(M, 1, 1)), f(nb(M, 1, -1)), f(nb(M, -1, 1)), f(nb(M, -1, -1))
    rules = {
        "aPP": e, "aMM": wv, "bPP": n, "bMM": s,
        "aPn": n | ne, "bPe": e | ne, "bMe": e | se, "aPs": s | se,
        "aMs": s | sw, "bMw": wv | sw, "bPw": wv | nw, "aMn": n | nw,
    }
    for k, cond in rules.items():
        w[k][marg & cond] = 0.0
    return w


def assemble_rhs(grid: Grid, cfg: Config, inp: Inputs, taud: np.ndarray) -> np.ndarray:
    """SSAFD::assemble_rhs, SSAFD.cc:282-417.  Returns (Mx, My, 2)."""
    dx, dy = grid.dx, grid.dy
    rho_i, rho_w, g = cfg.ice_density, cfg.sea_water_density, cfg.standard_gravity
    b = taud.copy()
    if cfg.calving_front_stress_boundary_condition:
        M = as_int(inp.mask)
        bb = cfg.ssa_dirichlet_bc
        f = m_ice_free_ocean if bb else m_ice_free
        aPP = np.where(f(nb(M, 1, 0)), 0, 1)
        aMM = np.where(f(nb(M, -1, 0)), 0, 1)
        bPP = np.where(f(nb(M, 0, 1)), 0, 1)
        bMM = np.where(f(nb(M, 0, -1)), 0, 1)
        H = inp.thickness
        bed = inp.bed
        H2 = H * H
        rho_g = rho_i * g
        with np.errstate(all="ignore"):
            grounded_term = np.where(bed >= cfg.sea_level, 0.5 * rho_g * H2,
                                     0.5 * rho_g * (H2 - (rho_w / rho_i) * np.power(cfg.sea_level - bed, 2.0)))
        ocean_pressure = np.where(m_ocean(M), 0.5 * rho_g * (1.0 - (rho_i / rho_w)) * H2, grounded_term)
        if inp.melange is not None:
            ocean_pressure = ocean_pressure * (1.0 - inp.melange)
        marg = is_marginal(M, bb)
        bu = taud[..., 0] + (aMM - aPP) * ocean_pressure / dx
        bv = taud[..., 1] + (bMM - bPP) * ocean_pressure / dy
        b[..., 0] = np.where(marg, bu, b[..., 0])
        b[..., 1] = np.where(marg, bv, b[..., 1])
        icefree = m_ice_free(M)
        b[icefree] = cfg.scaling * 0.0
    if inp.bc_mask is not None and inp.bc_values is not None:
        d = as_int(inp.bc_mask) == 1
        b[d, 0] = cfg.scaling * inp.bc_values[d, 0]
        b[d, 1] = cfg.scaling * inp.bc_values[d, 1]
    return b


# ---------------------------------------------------------------------------
# hardness, nu*H, beta
# ---------------------------------------------------------------------------
def hardness_staggered(grid: Grid, cfg: Config, inp: Inputs) -> np.ndarray:
    """SSAFD::compute_hardav_staggered (+ fracture_induced_softening), SSAFD.cc:1192-1310.

    Returns (Mx, My, 2): index 0 = east face (i+1/2, j), 1 = north face (i, j+1/2)."""
    H = inp.thickness
    M = as_int(inp.mask)
    icy = m_icy(M)
    out = np.zeros(H.shape + (2,))
    for o in range(2):
        oi, oj = 1 - o, o
        Hn = nb(H, oi, oj)
        icyn = nb(icy, oi, oj)
        Hf = np.where(icy & icyn, 0.5 * (H + Hn), np.where(icy, H, Hn))
        if cfg.flow_law == "isothermal_glen":
            B = averaged_hardness(cfg, Hf.ravel(), None, None).reshape(H.shape)
        else:
            E = inp.enthalpy
            Ef = 0.5 * (E + nb(E, oi, oj))
            B = averaged_hardness(cfg, Hf.ravel(), np.asarray(grid.z),
                                  Ef.reshape(-1, E.shape[2])).reshape(H.shape)
        out[..., o] = np.where(Hf == 0, -1e6, B)
    if cfg.do_fracture_density and inp.fracture_density is not None:
        n = cfg.ssa_Glen_exponent
        eps = cfg.fracture_density_softening_lower_limit
        D = inp.fracture_density
        for o in range(2):
            oi, oj = 1 - o, o
            phi = 0.5 * (D + nb(D, oi, oj))
            soft = np.power(1.0 - (1.0 - eps) * phi, -n)
            out[..., o] *= np.power(soft, -1.0 / n)
    return out


def notional_strength(cfg: Config) -> float:
    """SSAStrengthExtension::get_notional_strength, SSA.cc:61-63."""
    return cfg.constant_nu_strength_extension_ssa * cfg.min_thickness_strength_extension_ssa


def nuH_staggered(grid: Grid, cfg: Config, inp: Inputs, hardness: np.ndarray,
                  vel: np.ndarray, reg: float) -> np.ndarray:
    """SSAFD::compute_nuH_staggered, SSAFD.cc:1359-1421."""
    n = cfg.ssa_Glen_exponent
    scal = 1.0 / cfg.ssa_enhancement_factor ** (1.0 / n)
    dx, dy = grid.dx, grid.dy
    H = inp.thickness
    u, v = vel[..., 0], vel[..., 1]
    out = np.zeros(H.shape + (2,))
    for o in range(2):
        oi, oj = 1 - o, o
        Hf = 0.5 * (H + nb(H, oi, oj))
        if o == 0:
            u_x = (nb(u, 1, 0) - u) / dx
            u_y = (nb(u, 0, 1) + nb(u, 1, 1) - nb(u, 0, -1) - nb(u, 1, -1)) / (4 * dy)
            v_x = (nb(v, 1, 0) - v) / dx
            v_y = (nb(v, 0, 1) + nb(v, 1, 1) - nb(v, 0, -1) - nb(v, 1, -1)) / (4 * dy)
        else:
            u_x = (nb(u, 1, 0) + nb(u, 1, 1) - nb(u, -1, 0) - nb(u, -1, 1)) / (4 * dx)
            u_y = (nb(u, 0, 1) - u) / dy
            v_x = (nb(v, 1, 0) + nb(v, 1, 1) - nb(v, -1, 0) - nb(v, -1, 1)) / (4 * dx)
            v_y = (nb(v, 0, 1) - v) / dy
        nu = effective_viscosity(cfg, hardness[..., o], second_invariant_2d(u_x, u_y, v_x, v_y))
        r = nu * Hf
        r = r * scal
        r = r + reg
        out[..., o] = np.where(Hf < cfg.min_thickness_strength_extension_ssa, notional_strength(cfg), r)
    return out


def nuH_staggered_cfbc(grid: Grid, cfg: Config, inp: Inputs, hardness: np.ndarray,
                       vel: np.ndarray, reg: float) -> np.ndarray:
    """SSAFD::compute_nuH_staggered_cfbc, SSAFD.cc:1441-1582."""
    n = cfg.ssa_Glen_exponent
    scal = 1.0 / cfg.ssa_enhancement_factor ** (1.0 / n)
    dx, dy = grid.dx, grid.dy
    H = inp.thickness
    M = as_int(inp.mask)
    icy = m_icy(M)
    u, v = vel[..., 0], vel[..., 1]
    Hmin = cfg.min_thickness_strength_extension_ssa
    # m_work (SSAFD.cc:1463-1491), periodic everywhere
    wi = icy & nb(icy, 1, 0)
    wj = icy & nb(icy, 0, 1)
    U_X = np.where(wi, (nb(u, 1, 0) - u) / dx, 0.0)
    V_X = np.where(wi, (nb(v, 1, 0) - v) / dx, 0.0)
    W_I = np.where(wi, 1.0, 0.0)
    U_Y = np.where(wj, (nb(u, 0, 1) - u) / dy, 0.0)
    V_Y = np.where(wj, (nb(v, 0, 1) - v) / dy, 0.0)
    W_J = np.where(wj, 1.0, 0.0)
    out = np.zeros(H.shape + (2,))
    ns = notional_strength(cfg)
    # i-offset
    Hn = nb(H, 1, 0)
    Hf = np.where(wi, 0.5 * (H + Hn), np.where(icy, H, Hn))
    W = W_J + nb(W_J, 0, -1) + nb(W_J, 1, -1) + nb(W_J, 1, 0)
    with np.errstate(all="ignore"):
        u_y = np.where(W > 0, 1.0 / W * (U_Y + nb(U_Y, 0, -1) + nb(U_Y, 1, -1) + nb(U_Y, 1, 0)), 0.0)
        v_y = np.where(W > 0, 1.0 / W * (V_Y + nb(V_Y, 0, -1) + nb(V_Y, 1, -1) + nb(V_Y, 1, 0)), 0.0)
    nu = effective_viscosity(cfg, hardness[..., 0], second_invariant_2d(U_X, u_y, V_X, v_y))
    out[..., 0] = np.where(Hf >= Hmin, nu * Hf, ns)
    # j-offset
    Hn = nb(H, 0, 1)
    Hf = np.where(wj, 0.5 * (H + Hn), np.where(icy, H, Hn))
    W = W_I + nb(W_I, -1, 0) + nb(W_I, -1, 1) + nb(W_I, 0, 1)
    with np.errstate(all="ignore"):
        u_x = np.where(W > 0, 1.0 / W * (U_X + nb(U_X, -1, 0) + nb(U_X, -1, 1) + nb(U_X, 0, 1)), 0.0)
        v_x = np.where(W > 0, 1.0 / W * (V_X + nb(V_X, -1, 0) + nb(V_X, -1, 1) + nb(V_X, 0, 1)), 0.0)
    nu = effective_viscosity(cfg, hardness[..., 1], second_invariant_2d(u_x, U_Y, v_x, V_Y))
    out[..., 1] = np.where(Hf >= Hmin, nu * Hf, ns)
    out = out * scal
    out = out + reg
    return out


def compute_nuH(grid, cfg, inp, hardness, vel, reg):
    if cfg.calving_front_stress_boundary_condition:
        return nuH_staggered_cfbc(grid, cfg, inp, hardness, vel, reg)
    return nuH_staggered(grid, cfg, inp, hardness, vel, reg)


def beta_field(cfg: Config, inp: Inputs, vel: np.ndarray) -> np.ndarray:
    """Basal drag coefficient added to the diagonal, SSAFD.cc:744-763."""
    M = as_int(inp.mask)
    drag = basal_drag(cfg, inp.tauc, vel[..., 0], vel[..., 1])
    beta = np.where(m_grounded_ice(M), drag, np.where(m_ice_free_land(M), cfg.beta_ice_free_bedrock, 0.0))
    if cfg.sub_groundingline:
        beta = np.where(m_icy(M), inp.gl_mask * drag, beta)
    return beta


def nuH_norm(grid: Grid, nuH: np.ndarray, nuH_old: np.ndarray):
    """SSAFD::compute_nuH_norm, SSAFD.cc:1170-1189.

    The L1 norms run over the ghosted local vectors (stencil width 1, one rank),
    i.e. every cell is counted once plus once per periodic ghost copy of it."""
    Mx, My = nuH.shape[:2]
    wi = np.ones(Mx)
    wj = np.ones(My)
    wi[0] += 1
    wi[Mx - 1] += 1
    wj[0] += 1
    wj[My - 1] += 1
    w = np.outer(wi, wj)[..., None]
    area = grid.dx * grid.dy
    d = nuH_old - nuH          # nuH_old.add(-1, nuH)
    nuNorm = (np.abs(nuH) * w).reshape(-1, 2).sum(axis=0) * area
    nuChange = (np.abs(d) * w).reshape(-1, 2).sum(axis=0) * area
    return math.sqrt(nuNorm[0] ** 2 + nuNorm[1] ** 2), math.sqrt(nuChange[0] ** 2 + nuChange[1] ** 2)


# ---------------------------------------------------------------------------
# matrix
# ---------------------------------------------------------------------------
class ZeroDiagonal(RuntimeError):
    pass


def stencil_coefficients(grid: Grid, cfg: Config, inp: Inputs, nuH: np.ndarray,
                         beta: np.ndarray):
    """Per-cell eq1/eq2 coefficient arrays of SSAFD::assemble_matrix (SSAFD.cc:540-796).

    Returns (eq1, eq2, diag_only) with eq*: (18, Mx, My); entries 0-8 multiply u at
    (i-1..i+1, j+1..j-1) row-major as in the reference's I/J tables, 9-17 multiply v.
    ``diag_only`` marks Dirichlet / CFBC ice-free rows whose only entry is m_scaling."""
    dx, dy = grid.dx, grid.dy
    M = as_int(inp.mask)
    c_w = nb(nuH[..., 0], -1, 0)
    c_e = nuH[..., 0].copy()
    c_s = nb(nuH[..., 1], 0, -1)
    c_n = nuH[..., 1].copy()
    if cfg.nu_bedrock_set:
        H, bed, srf = inp.thickness, inp.bed, inp.surface
        nbb = cfg.nu_bedrock
        thick = H > 0.0
        c_w = np.where(thick & (nb(bed, -1, 0) > srf) & m_ice_free_land(nb(M, -1, 0)),
                       nbb * 0.5 * (H + nb(H, -1, 0)), c_w)
        c_e = np.where(thick & (nb(bed, 1, 0) > srf) & m_ice_free_land(nb(M, 1, 0)),
                       nbb * 0.5 * (H + nb(H, 1, 0)), c_e)
        c_n = np.where(thick & (nb(bed, 0, 1) > srf) & m_ice_free_land(nb(M, 0, 1)),
                       nbb * 0.5 * (H + nb(H, 0, 1)), c_n)
        # SSAFD.cc:582 uses thickness(i+1, j) here (sic)
        c_s = np.where(thick & (nb(bed, 0, -1) > srf) & m_ice_free_land(nb(M, 0, -1)),
                       nbb * 0.5 * (H + nb(H, 1, 0)), c_s)
    w = cfbc_weights(M, cfg)
    aMn, aPn, aMM, aPP, aMs, aPs = w["aMn"], w["aPn"], w["aMM"], w["aPP"], w["aMs"], w["aPs"]
    bPw, bPP, bPe, bMw, bMM, bMe = w["bPw"], w["bPP"], w["bPe"], w["bMw"], w["bMM"], w["bMe"]
    dx2, dy2, d4, d2 = dx * dx, dy * dy, 4 * dx * dy, 2 * dx * dy
    Z = np.zeros(M.shape)
    eq1 = [
        Z, -c_n * bPP / dy2, Z,
        -4 * c_w * aMM / dx2, (c_n * bPP + c_s * bMM) / dy2 + (4 * c_e * aPP + 4 * c_w * aMM) / dx2, -4 * c_e * aPP / dx2,
        Z, -c_s * bMM / dy2, Z,
        c_w * aMM * bPw / d2 + c_n * aMn * bPP / d4,
        (c_n * aPn * bPP - c_n * aMn * bPP) / d4 + (c_w * aMM * bPP - c_e * aPP * bPP) / d2,
        -c_e * aPP * bPe / d2 - c_n * aPn * bPP / d4,
        (c_w * aMM * bMw - c_w * aMM * bPw) / d2 + (c_n * aMM * bPP - c_s * aMM * bMM) / d4,
        (c_n * aPP * bPP - c_n * aMM * bPP - c_s * aPP * bMM + c_s * aMM * bMM) / d4
        + (c_e * aPP * bPP - c_w * aMM * bPP - c_e * aPP * bMM + c_w * aMM * bMM) / d2,
        (c_e * aPP * bPe - c_e * aPP * bMe) / d2 + (c_s * aPP * bMM - c_n * aPP * bPP) / d4,
        -c_w * aMM * bMw / d2 - c_s * aMs * bMM / d4,
        (c_s * aMs * bMM - c_s * aPs * bMM) / d4 + (c_e * aPP * bMM - c_w * aMM * bMM) / d2,
        c_e * aPP * bMe / d2 + c_s * aPs * bMM / d4,
    ]
    eq2 = [
        c_w * aMM * bPw / d4 + c_n * aMn * bPP / d2,
        (c_n * aPn * bPP - c_n * aMn * bPP) / d2 + (c_w * aMM * bPP - c_e * aPP * bPP) / d4,
        -c_e * aPP * bPe / d4 - c_n * aPn * bPP / d2,
        (c_w * aMM * bMw - c_w * aMM * bPw) / d4 + (c_n * aMM * bPP - c_s * aMM * bMM) / d2,
        (c_n * aPP * bPP - c_n * aMM * bPP - c_s * aPP * bMM + c_s * aMM * bMM) / d2
        + (c_e * aPP * bPP - c_w * aMM * bPP - c_e * aPP * bMM + c_w * aMM * bMM) / d4,
        (c_e * aPP * bPe - c_e * aPP * bMe) / d4 + (c_s * aPP * bMM - c_n * aPP * bPP) / d2,
        -c_w * aMM * bMw / d4 - c_s * aMs * bMM / d2,
        (c_s * aMs * bMM - c_s * aPs * bMM) / d2 + (c_e * aPP * bMM - c_w * aMM * bMM) / d4,
        c_e * aPP * bMe / d4 + c_s * aPs * bMM / d2,
        Z, -4 * c_n * bPP / dy2, Z,
        -c_w * aMM / dx2, (4 * c_n * bPP + 4 * c_s * bMM) / dy2 + (c_e * aPP + c_w * aMM) / dx2, -c_e * aPP / dx2,
        Z, -4 * c_s * bMM / dy2, Z,
    ]
    eq1 = np.array([np.broadcast_to(a, M.shape) for a in eq1])
    eq2 = np.array([np.broadcast_to(a, M.shape) for a in eq2])
    eq1[4] = eq1[4] + beta
    eq2[13] = eq2[13] + beta

    diag_only = np.zeros(M.shape, dtype=bool)
    if inp.bc_mask is not None and inp.bc_values is not None:
        diag_only |= as_int(inp.bc_mask) == 1
    if cfg.calving_front_stress_boundary_condition:
        diag_only |= m_ice_free(M)
    return eq1, eq2, diag_only


# (I, J) offsets of the 18 stencil entries, SSAFD.cc:710-737
STENCIL_DI = np.array([-1, 0, 1] * 6)
STENCIL_DJ = np.array([1, 1, 1, 0, 0, 0, -1, -1, -1] * 2)
STENCIL_C = np.array([0] * 9 + [1] * 9)


def assemble_matrix(grid: Grid, cfg: Config, inp: Inputs, nuH, beta, check_diagonal=True):
    """SSAFD::assemble_matrix, SSAFD.cc:496-811, as a scipy CSR matrix.

    Unknown index: 2 * (i * My + j) + c (j contiguous, u/v interleaved)."""
    Mx, My = grid.Mx, grid.My
    if Mx < 3 or My < 3:
        raise ValueError("grids narrower than 3 cells alias stencil columns; not supported")
    eq1, eq2, diag_only = stencil_coefficients(grid, cfg, inp, nuH, beta)
    if check_diagonal:
        eps = 1e-16
        bad1 = (np.abs(eq1[4]) < eps) & ~diag_only
        bad2 = (np.abs(eq2[13]) < eps) & ~diag_only
        if bad1.any() or bad2.any():
            i, j = np.argwhere(bad1 | bad2)[0]
            raise ZeroDiagonal(f"zero diagonal entry at a regular location: i = {i}, j = {j}")
    I, J = np.meshgrid(np.arange(Mx), np.arange(My), indexing="ij")
    cell = I * My + J
    rows, cols, vals = [], [], []
    for m in range(18):
        ci = (I + STENCIL_DI[m]) % Mx
        cj = (J + STENCIL_DJ[m]) % My
        col = 2 * (ci * My + cj) + STENCIL_C[m]
        for c, eq in ((0, eq1), (1, eq2)):
            v = np.where(diag_only, 0.0, eq[m])
            rows.append((2 * cell + c).ravel())
            cols.append(col.ravel())
            vals.append(v.ravel())
    # Dirichlet / ice-free rows: the scaled identity (SSAFD.cc:1620-1641)
    d = diag_only.ravel()
    idx = cell.ravel()[d]
    for c in range(2):
        rows.append(2 * idx + c)
        cols.append(2 * idx + c)
        vals.append(np.full(idx.shape, cfg.scaling))
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(2 * Mx * My, 2 * Mx * My)).tocsr()
    A.sum_duplicates()
    return A


def apply_stencil(grid: Grid, cfg: Config, inp: Inputs, nuH, beta, x: np.ndarray) -> np.ndarray:
    """y = A x computed stencil-wise (same arithmetic as assemble_matrix, no sparse matrix)."""
    eq1, eq2, diag_only = stencil_coefficients(grid, cfg, inp, nuH, beta)
    y = np.zeros_like(x)
    for m in range(18):
        xm = nb(x[..., STENCIL_C[m]], STENCIL_DI[m], STENCIL_DJ[m])
        y[..., 0] += eq1[m] * xm
        y[..., 1] += eq2[m] * xm
    y[diag_only] = cfg.scaling * x[diag_only]
    return y


def line_block_part(grid: Grid, A):
    """The line block-Jacobi preconditioner's matrix M: the entries of A (unknown index
    2 * (i * My + j) + c) that couple a cell to itself and to its neighbours j - 1 and
    j + 1 on the same grid line of constant i; the couplings across the line's two ends
    (the periodic wrap) and between lines are dropped.  No reference counterpart: it
    stands in for the ILU(0) of PETSc's default block Jacobi (SSAFD.cc:136-161)."""
    A = A.tocoo()
    My = grid.My
    rc, cc = A.row // 2, A.col // 2
    keep = (rc // My == cc // My) & (np.abs(rc % My - cc % My) <= 1)
    return sp.csr_matrix((A.data[keep], (A.row[keep], A.col[keep])), shape=A.shape)


def line_block_solve(grid: Grid, A, r: np.ndarray) -> np.ndarray:
    """z = M^-1 r for M = line_block_part(grid, A), by a sparse direct solve."""
    M = line_block_part(grid, A).tocsc()
    return spla.spsolve(M, r.ravel()).reshape(r.shape)


def line_block_lu_solve(grid: Grid, A, r: np.ndarray) -> np.ndarray:
    """The same z by the per-line block LU recurrences (pure Python, small grids):
    P_j = (D_j - L_j G_{j-1})^-1, F_j = -P_j L_j, G_j = P_j U_j;
    y_j = P_j r_j + F_j y_{j-1};  z_j = y_j - G_j z_{j+1}."""
    Mx, My = grid.Mx, grid.My
    A = A.tocsr()

    def block(k, kk):
        return A[2 * k:2 * k + 2, 2 * kk:2 * kk + 2].toarray()

    z = np.zeros((Mx, My, 2))
    for i in range(Mx):
        G, y = [], []
        Gp, yp = np.zeros((2, 2)), np.zeros(2)
        for j in range(My):
            k = i * My + j
            Lb = block(k, k - 1) if j > 0 else np.zeros((2, 2))
            U = block(k, k + 1) if j < My - 1 else np.zeros((2, 2))
            Pj = np.linalg.inv(block(k, k) - Lb @ Gp)
            Gp = Pj @ U
            yp = Pj @ r[i, j] - Pj @ Lb @ yp
            G.append(Gp)
            y.append(yp)
        x = np.zeros(2)
        for j in range(My - 1, -1, -1):
            x = y[j] - G[j] @ x
            z[i, j] = x
    return z


# ---------------------------------------------------------------------------
# Picard loop and recovery strategies
# ---------------------------------------------------------------------------
class KSPFailure(RuntimeError):
    pass


class PicardFailure(RuntimeError):
    pass


@dataclass
class SolveStats:
    picard_iterations: int = 0
    strategy: int = 0            # 0 default, 1 under-relaxation, 2 over-regularization
    converged: bool = False
    nuH_norm: float = 0.0
    nuH_norm_change: float = 0.0
    history: list = field(default_factory=list)


def linear_solve(A, b, x0, method="direct", rtol=1e-12, grid=None, nranks=1, nthreads=0):
    if method == "petsc":
        x, its, reason = petsc_gmres_bjacobi(A, b, x0, grid.Mx, grid.My, nranks=nranks, rtol=rtol,
                                             nthreads=nthreads)
        if reason < 0:
            raise KSPFailure(f"KSP diverged, reason {reason}")
        return x
    if method == "direct":
        lu = spla.splu(A.tocsc())
        return lu.solve(b)
    if method == "ilu_gmres":
        ilu = spla.spilu(A.tocsc(), fill_factor=1, drop_tol=0.0)
        Mop = spla.LinearOperator(A.shape, ilu.solve)
        x, info = spla.gmres(A, b, x0=x0, M=Mop, restart=30, rtol=rtol, maxiter=10000)
        if info != 0:
            raise KSPFailure(f"gmres info={info}")
        return x
    raise ValueError(method)


class SSAFDOracle:
    """CPU restatement of SSAFD::solve and its strategy ladder (SSAFD.cc:869-1155)."""

    def __init__(self, grid: Grid, cfg: Config, inp: Inputs, linear="direct", ksp_rtol=1e-12,
                 nranks=1, nthreads=0):
        self.nranks = nranks
        self.nthreads = nthreads
        self.grid = grid
        self.cfg = cfg
        self.inp = inp
        self.linear = linear
        self.ksp_rtol = ksp_rtol
        self.velocity = np.zeros((grid.Mx, grid.My, 2))
        self.taud = None
        self.b = None
        self.hardness = None
        self.nuH = None
        self.stats = SolveStats()

    def set_initial_guess(self, v):
        self.velocity = np.array(v, dtype=np.float64).reshape(self.grid.Mx, self.grid.My, 2)

    def prepare(self):
        g, c, i = self.grid, self.cfg, self.inp
        self.taud = driving_stress(g, c, i)
        self.b = assemble_rhs(g, c, i, self.taud)
        self.hardness = hardness_staggered(g, c, i)

    def picard_manager(self, reg, underrelax):
        g, c, i = self.grid, self.cfg, self.inp
        vel = self.velocity.copy()
        nuH = compute_nuH(g, c, i, self.hardness, vel, reg)
        for k in range(c.max_iterations_ssafd):
            nuH_old = nuH.copy()
            beta = beta_field(c, i, vel)
            A = assemble_matrix(g, c, i, nuH, beta)
            x = linear_solve(A, self.b.ravel(), vel.ravel(), self.linear, self.ksp_rtol, g,
                             self.nranks, self.nthreads)
            vel = x.reshape(vel.shape)
            self.velocity = vel
            nuH = compute_nuH(g, c, i, self.hardness, vel, reg)
            if underrelax != 1.0:
                nuH = nuH * underrelax
                nuH = nuH + (1.0 - underrelax) * nuH_old
            norm, change = nuH_norm(g, nuH, nuH_old)
            self.nuH = nuH
            self.stats.history.append((norm, change))
            self.stats.picard_iterations = k + 1
            self.stats.nuH_norm, self.stats.nuH_norm_change = norm, change
            if norm == 0 or change / norm < c.ssafd_relative_convergence:
                return
        raise PicardFailure("effective viscosity not converged")

    def solve(self):
        """SSAFD::solve, SSAFD.cc:869-924 (the k < 3 loop exits silently if every strategy fails)."""
        velocity_old = self.velocity.copy()
        self.prepare()
        c = self.cfg
        self.stats = SolveStats()
        for k in range(3):
            try:
                self.stats.strategy = k
                if k == 0:
                    self.picard_manager(c.epsilon_ssa, 1.0)
                elif k == 1:
                    self.picard_manager(c.epsilon_ssa, c.ssafd_nuH_iter_failure_underrelaxation)
                else:
                    self.picard_strategy_regularization(velocity_old)
                self.stats.converged = True
                break
            except PicardFailure:
                continue
        if c.brutal_sliding:
            self.velocity = self.velocity * c.brutal_sliding_scale
        return self.velocity

    def picard_strategy_regularization(self, velocity_old):
        """SSAFD.cc:1122-1155."""
        reg = self.cfg.epsilon_ssa
        if reg <= 0.0:
            raise PicardFailure("will not attempt over-regularization of nuH because nuH_regularization == 0.0.")
        for k in range(5):
            self.velocity = velocity_old.copy()
            reg *= 4.0
            try:
                self.picard_manager(reg, 1.0)
                return
            except PicardFailure:
                if k == 4:
                    raise PicardFailure("exceeded the max. number of nuH over-regularization attempts")


def basal_frictional_heating(cfg: Config, inp: Inputs, vel):
    """ShallowStressBalance::compute_basal_frictional_heating, ShallowStressBalance.cc:179-205."""
    M = as_int(inp.mask)
    u, v = vel[..., 0], vel[..., 1]
    C = basal_drag(cfg, inp.tauc, u, v)
    bx, by = -C * u, -C * v
    return np.where(m_ocean(M), 0.0, -bx * u - by * v)


# ---------------------------------------------------------------------------
# the consumers of the SSA velocity in StressBalance::update (full update)
# ---------------------------------------------------------------------------
def _margin_differences(grid: Grid, M):
    """The one-sided / centred difference weights at ice margins shared by the vertical
    velocity and the strain heating (PISMStressBalance.cc:229-257, 414-442): (west, east,
    D_x, south, north, D_y) per cell."""
    icy, free = m_icy(M), m_ice_free(M)

    def cut(di, dj):
        Mn_icy, Mn_free = nb(icy, di, dj), nb(free, di, dj)
        return np.where((icy & Mn_free) | (free & Mn_icy), 0.0, 1.0)

    east, west, north, south = cut(1, 0), cut(-1, 0), cut(0, 1), cut(0, -1)
    D_x = np.where(east + west > 0, 1.0 / (grid.dx * np.maximum(east + west, 1.0)), 0.0)
    D_y = np.where(north + south > 0, 1.0 / (grid.dy * np.maximum(north + south, 1.0)), 0.0)
    return west, east, D_x, south, north, D_y


def constant_in_column(vel, Mz: int):
    """ConstantInColumn::update, SSB_Modifier.cc:126-152: every level of the 3-D horizontal
    velocity is the column's SSA velocity.  Returns (u3, v3), (Mx, My, Mz)."""
    u3 = np.repeat(vel[..., 0:1], Mz, axis=2)
    v3 = np.repeat(vel[..., 1:2], Mz, axis=2)
    return u3, v3


def vertical_velocity(grid: Grid, inp: Inputs, u3, v3, basal_melt_rate=None):
    """StressBalance::compute_vertical_velocity, PISMStressBalance.cc:192-287: the trapezoid
    rule integral of -(u_x + v_y) up each column from w(0) = -basal melt rate (or 0), with
    one-sided differences at ice margins."""
    M = as_int(inp.mask)
    west, east, D_x, south, north, D_y = _margin_differences(grid, M)
    z = np.asarray(grid.z, dtype=np.float64)
    Mz = len(z)
    w = np.zeros(u3.shape)
    w[..., 0] = 0.0 if basal_melt_rate is None else -np.asarray(basal_melt_rate, dtype=np.float64)

    def integrand(k):
        u_x = D_x * (west * (u3[..., k] - nb(u3[..., k], -1, 0)) + east * (nb(u3[..., k], 1, 0) - u3[..., k]))
        v_y = D_y * (south * (v3[..., k] - nb(v3[..., k], 0, -1)) + north * (nb(v3[..., k], 0, 1) - v3[..., k]))
        return u_x + v_y

    old = integrand(0)
    for k in range(1, Mz):
        new = integrand(k)
        w[..., k] = w[..., k - 1] - 0.5 * (new + old) * (z[k] - z[k - 1])
        old = new
    return w


def volumetric_strain_heating(grid: Grid, cfg: Config, inp: Inputs, u3, v3):
    """StressBalance::compute_volumetric_strain_heating, PISMStressBalance.cc:369-499:
    Sigma = 2 e^(-1/n) B(E, p) D^(1/n + 1) with the shallow approximation of D^2 (D2,
    PISMStressBalance.cc:309-311) at the levels k <= kBelowHeight(H), zero above."""
    M = as_int(inp.mask)
    west, east, D_x, south, north, D_y = _margin_differences(grid, M)
    z = np.asarray(grid.z, dtype=np.float64)
    Mz = len(z)
    H = np.asarray(inp.thickness, dtype=np.float64)
    ks = k_below_height(z, H)
    n = cfg.ssa_Glen_exponent
    exponent = 0.5 * (1.0 / n + 1.0)
    e_to_a_power = cfg.ssa_enhancement_factor ** (-1.0 / n)
    # an isothermal flow law reads no enthalpy
    E = np.zeros(u3.shape) if inp.enthalpy is None else np.asarray(inp.enthalpy, dtype=np.float64)
    sigma = np.zeros(u3.shape)
    for k in range(Mz - 1):
        uk, vk = u3[..., k], v3[..., k]
        u_x = D_x * (west * (uk - nb(uk, -1, 0)) + east * (nb(uk, 1, 0) - uk))
        u_y = D_y * (south * (uk - nb(uk, 0, -1)) + north * (nb(uk, 0, 1) - uk))
        v_x = D_x * (west * (vk - nb(vk, -1, 0)) + east * (nb(vk, 1, 0) - vk))
        v_y = D_y * (south * (vk - nb(vk, 0, -1)) + north * (nb(vk, 0, 1) - vk))
        if k > 0:
            dz = z[k + 1] - z[k - 1]
            u_z = (u3[..., k + 1] - u3[..., k - 1]) / dz
            v_z = (v3[..., k + 1] - v3[..., k - 1]) / dz
        else:
            dz = z[1] - z[0]
            u_z = (u3[..., 1] - u3[..., 0]) / dz
            v_z = (v3[..., 1] - v3[..., 0]) / dz
        B = hardness_parameter(cfg, E[..., k], ec_pressure(cfg, H - z[k]))
        D2 = 0.5 * ((u_x + v_y) ** 2 + u_x * u_x + v_y * v_y + 0.5 * ((u_y + v_x) ** 2 + u_z * u_z + v_z * v_z))
        sigma[..., k] = np.where(k <= ks, 2.0 * e_to_a_power * B * np.power(D2, exponent), 0.0)
    return sigma


# ---------------------------------------------------------------------------
# mass transport consuming the SSA velocity: IceModel::massContExplicitStep
# ---------------------------------------------------------------------------
MASS_TOTALS = ("grounded_basal_ice_flux", "nonneg_rule_flux", "sub_shelf_ice_flux", "surface_ice_flux",
               "sum_divQ_SIA", "sum_divQ_SSA", "Href_to_H_flux", "H_to_Href_flux")


def cell_interface_velocities(cfg: Config, inp: Inputs, vel):
    """IceModel::cell_interface_fluxes, iMgeometry.cc:309-410 (the SSA part): the normal
    velocity at the four faces of each cell, (e, w, n, s), by the icy / ice-free cases of the
    two cells and, with ssa_dirichlet_bc, the boundary-condition cases."""
    M = as_int(inp.mask)
    icy = m_icy(M)
    u, v = vel[..., 0], vel[..., 1]
    out = {}
    for name, di, dj, comp in (("e", 1, 0, u), ("w", -1, 0, u), ("n", 0, 1, v), ("s", 0, -1, v)):
        icy_n = nb(icy, di, dj)
        comp_n = nb(comp, di, dj)
        f = np.where(icy & icy_n, 0.5 * (comp + comp_n),
                     np.where(icy & ~icy_n, comp, np.where(~icy & icy_n, comp_n, 0.0)))
        if cfg.ssa_dirichlet_bc and inp.bc_mask is not None:
            bm = as_int(inp.bc_mask)
            bm_n = nb(bm, di, dj)
            bv = inp.bc_values[..., 0 if comp is u else 1]
            bv_n = nb(bv, di, dj)
            f = np.where((bm == 1) & (bm_n == 1), 0.5 * (bv + bv_n),
                         np.where((bm == 1) & (bm_n == 0), bv, np.where((bm == 0) & (bm_n == 1), bv_n, f)))
        out[name] = f
    return out


def mass_continuity_step(grid: Grid, cfg: Config, inp: Inputs, vel, dt, climatic_mass_balance,
                         basal_melt_rate=None, cell_area=None):
    """IceModel::massContExplicitStep, iMgeometry.cc:497-819, with the ConstantInColumn
    modifier (no diffusive flux: divQ_SIA = 0), part_grid off and no residual redistribution:
    upwinded SSA flux divergence, surface and basal mass balance (zero on ice-free ocean and at
    Dirichlet locations), the non-negativity rule, and the eight flux totals in kg.  Returns
    (new thickness, flux divergence, totals)."""
    M = as_int(inp.mask)
    H = np.asarray(inp.thickness, dtype=np.float64)
    dx, dy = grid.dx, grid.dy
    rho = cfg.ice_density
    area = np.full(H.shape, dx * dy) if cell_area is None else np.asarray(cell_area, dtype=np.float64)
    meter_to_kg = area * rho
    meter_per_s_to_kg = meter_to_kg * dt
    f = cell_interface_velocities(cfg, inp, vel)
    divQ_SIA = np.zeros(H.shape)   # (Q.e - Q.w) / dx + (Q.n - Q.s) / dy with Q = 0
    divQ_SSA = 0.0 + (f["e"] * np.where(f["e"] > 0, H, nb(H, 1, 0))
                      - f["w"] * np.where(f["w"] > 0, nb(H, -1, 0), H)) / dx
    divQ_SSA = divQ_SSA + (f["n"] * np.where(f["n"] > 0, H, nb(H, 0, 1))
                           - f["s"] * np.where(f["s"] > 0, nb(H, 0, -1), H)) / dy
    smb = np.asarray(climatic_mass_balance, dtype=np.float64) / rho
    bmr = np.zeros(H.shape) if basal_melt_rate is None else np.asarray(basal_melt_rate, dtype=np.float64)
    free_ocean = m_ice_free_ocean(M)
    smb = np.where(free_ocean, 0.0, smb)
    bmr = np.where(free_ocean, 0.0, bmr)
    href_to_h = np.zeros(H.shape)
    if cfg.ssa_dirichlet_bc and inp.bc_mask is not None:
        bc = as_int(inp.bc_mask) == 1
        smb, bmr = np.where(bc, 0.0, smb), np.where(bc, 0.0, bmr)
        href_to_h = np.where(bc, 0.0, href_to_h)
        divQ_SIA, divQ_SSA = np.where(bc, 0.0, divQ_SIA), np.where(bc, 0.0, divQ_SSA)
    flux_divergence = divQ_SIA + divQ_SSA
    Hnew = H + (dt * (smb - bmr - (divQ_SIA + divQ_SSA)) + href_to_h)
    nonneg = np.where(Hnew < 0.0, -Hnew, 0.0)
    Hnew = np.where(Hnew < 0.0, 0.0, Hnew)
    grounded = m_grounded(M)
    totals = {
        "grounded_basal_ice_flux": float(np.sum(np.where(grounded, -bmr * meter_per_s_to_kg, 0.0))),
        "nonneg_rule_flux": float(np.sum(nonneg * meter_to_kg)),
        "sub_shelf_ice_flux": float(np.sum(np.where(grounded, 0.0, -bmr * meter_per_s_to_kg))),
        "surface_ice_flux": float(np.sum(smb * meter_per_s_to_kg)),
        "sum_divQ_SIA": float(np.sum(-divQ_SIA * meter_per_s_to_kg)),
        "sum_divQ_SSA": float(np.sum(-divQ_SSA * meter_per_s_to_kg)),
        "Href_to_H_flux": float(np.sum(href_to_h * meter_to_kg)),
        "H_to_Href_flux": 0.0,
    }
    return Hnew, flux_divergence, totals


# ---------------------------------------------------------------------------
# strain rates and 2-D stresses of the SSA velocity; eigen-calving
# ---------------------------------------------------------------------------
def _velocity_gradient(grid: Grid, M, vel):
    """u_x, u_y, v_x, v_y of ShallowStressBalance.cc:249-293 (and :330-371): centred
    differences written as weighted one-sided ones, a side dropped where that neighbour is
    ice-free, the derivative zero where both are."""
    free = m_ice_free(M)
    east, west = np.where(nb(free, 1, 0), 0.0, 1.0), np.where(nb(free, -1, 0), 0.0, 1.0)
    north, south = np.where(nb(free, 0, 1), 0.0, 1.0), np.where(nb(free, 0, -1), 0.0, 1.0)
    u, v = vel[..., 0], vel[..., 1]
    with np.errstate(divide="ignore", invalid="ignore"):
        rx = np.where(west + east > 0, 1.0 / (grid.dx * (west + east)), 0.0)
        ry = np.where(south + north > 0, 1.0 / (grid.dy * (south + north)), 0.0)
    u_x = np.where(west + east > 0, rx * (west * (u - nb(u, -1, 0)) + east * (nb(u, 1, 0) - u)), 0.0)
    v_x = np.where(west + east > 0, rx * (west * (v - nb(v, -1, 0)) + east * (nb(v, 1, 0) - v)), 0.0)
    u_y = np.where(south + north > 0, ry * (south * (u - nb(u, 0, -1)) + north * (nb(u, 0, 1) - u)), 0.0)
    v_y = np.where(south + north > 0, ry * (south * (v - nb(v, 0, -1)) + north * (nb(v, 0, 1) - v)), 0.0)
    return u_x, u_y, v_x, v_y


def principal_strain_rates(grid: Grid, mask, vel):
    """ShallowStressBalance::compute_2D_principal_strain_rates, ShallowStressBalance.cc:224-305:
    the eigenvalues (max, min) of the vertically integrated horizontal strain rate tensor,
    zero on ice-free cells.  Returns [Mx, My, 2] (1/s)."""
    M = as_int(mask)
    u_x, u_y, v_x, v_y = _velocity_gradient(grid, M, vel)
    A = 0.5 * (u_x + v_y)
    B = 0.5 * (u_x - v_y)
    Dxy = 0.5 * (v_x + u_y)
    q = np.sqrt(B * B + Dxy * Dxy)
    free = m_ice_free(M)
    return np.stack([np.where(free, 0.0, A + q), np.where(free, 0.0, A - q)], axis=-1)


def deviatoric_stresses_2d(grid: Grid, cfg: Config, mask, vel):
    """ShallowStressBalance::compute_2D_stresses, ShallowStressBalance.cc:308-386: the
    effective viscosity of the constant hardness ice_softness^(-1/n) at the strain rate's
    second invariant, times (u_x, v_y, (u_y + v_x) / 2).  Returns [Mx, My, 3] (Pa)."""
    M = as_int(mask)
    u_x, u_y, v_x, v_y = _velocity_gradient(grid, M, vel)
    hardness = cfg.ice_softness ** (-1.0 / cfg.ssa_Glen_exponent)
    nu = effective_viscosity(cfg, hardness, second_invariant_2d(u_x, u_y, v_x, v_y))
    free = m_ice_free(M)
    return np.stack([np.where(free, 0.0, nu * u_x), np.where(free, 0.0, nu * v_y),
                     np.where(free, 0.0, 0.5 * nu * (u_y + v_x))], axis=-1)


EIGEN_CALVING_OFFSET = 2   # EigenCalving::m_stencil_width, PISMEigenCalving.cc:33


def _eigen_calving_front(grid: Grid, M, edot, K):
    """The calving front cells of EigenCalving (ice-free ocean next to floating ice) and their
    horizontal calving rate K eigen1 eigen2 (PISMEigenCalving.cc:115-176, 283-322): the
    principal strain rates averaged over the floating, non-margin cells two cells away, in
    the order (i-2, j), (i+2, j), (i, j-2), (i, j+2).  As one process runs it: a strain rate
    read across the grid's edge is the ghost value 0; the mask wraps periodically (the
    reference's mask ghosts are two wide, so a front cell within three cells of the edge
    reads beyond them in ice_margin).  Returns (front, calving law applies, rate)."""
    floating = m_floating_ice(M)
    free = m_ice_free(M)
    front = m_ice_free_ocean(M) & (nb(floating, 1, 0) | nb(floating, -1, 0) | nb(floating, 0, 1)
                                   | nb(floating, 0, -1))
    margin = m_icy(M) & (nb(free, 1, 0) | nb(free, -1, 0) | nb(free, 0, 1) | nb(free, 0, -1))
    use = floating & ~margin
    o = EIGEN_CALVING_OFFSET
    Mx, My = M.shape
    ii, jj = np.meshgrid(np.arange(Mx), np.arange(My), indexing="ij")
    e1, e2, cnt = np.zeros(M.shape), np.zeros(M.shape), np.zeros(M.shape)
    for di, dj in ((-o, 0), (o, 0), (0, -o), (0, o)):
        take = nb(use, di, dj)
        # the strain rates' ghosts are never refreshed after EigenCalving::init set them to 0
        inside = (ii + di >= 0) & (ii + di < Mx) & (jj + dj >= 0) & (jj + dj < My)
        e1 = e1 + np.where(take, np.where(inside, nb(edot[..., 0], di, dj), 0.0), 0.0)
        e2 = e2 + np.where(take, np.where(inside, nb(edot[..., 1], di, dj), 0.0), 0.0)
        cnt = cnt + take
    e1 = np.where(cnt > 0, e1 / np.maximum(cnt, 1), e1)
    e2 = np.where(cnt > 0, e2 / np.maximum(cnt, 1), e2)
    law = front & (e2 > 0.0) & (e1 > 0.0)
    return front, law, np.where(law, K * e1 * (e2 - 0.0), 0.0)


def remove_narrow_tongues(M, H):
    """EigenCalving::remove_narrow_tongues, PISMEigenCalving.cc:420-493, as one process runs it:
    cells in (i, j) order with i outer (IceGrid.hh:335-345), the mask updated in place, so a
    neighbour earlier in that order and inside the grid is read after its own update, while
    one across the periodic edge is read from the ghost copy made before the loop.  Returns
    the new (mask, thickness)."""
    M0 = np.asarray(M, dtype=np.int64).copy()
    live = M0.copy()
    H = np.asarray(H, dtype=np.float64).copy()
    Mx, My = M0.shape

    def at(i, j):
        if 0 <= i < Mx and 0 <= j < My:
            return live[i, j]
        return M0[i % Mx, j % My]

    for i in range(Mx):
        for j in range(My):
            m = live[i, j]
            if not (m == MASK_GROUNDED or m == MASK_FLOATING):
                continue
            if m == MASK_GROUNDED:
                test = lambda a: a == MASK_ICE_FREE_OCEAN   # noqa: E731 (ice_free_ocean, Mask.hh:59-61)
            else:
                test = lambda a: not (a == MASK_GROUNDED or a == MASK_FLOATING)   # noqa: E731 (ice_free)
            N, E, S, W = test(at(i, j + 1)), test(at(i + 1, j)), test(at(i, j - 1)), test(at(i - 1, j))
            NE, NW, SE, SW = test(at(i + 1, j + 1)), test(at(i - 1, j + 1)), test(at(i + 1, j - 1)), test(at(i - 1, j - 1))
            if ((not W and NW and SW and N and S and E) or (not N and NW and NE and W and E and S)
                    or (not E and NE and SE and W and S and N) or (not S and SW and SE and W and E and N)):
                live[i, j] = MASK_ICE_FREE_OCEAN
                H[i, j] = 0.0
    return live, H


def eigen_calving(grid: Grid, mask, Href, thickness, vel, dt, K):
    """EigenCalving::update, PISMEigenCalving.cc:77-235: the principal strain rates of the
    velocity on this mask; at each calving front cell the calving rate K e1 e2 H_average / dx
    lowers Href and, where Href goes negative, the loss is shared among the floating
    neighbours, which are cut (thickness 0, ice-free ocean, Href = max(H - loss, 0)); then
    remove_narrow_tongues.  Returns (mask, Href, thickness)."""
    M = as_int(mask)
    H = np.asarray(thickness, dtype=np.float64).copy()
    Href = np.asarray(Href, dtype=np.float64).copy()
    edot = principal_strain_rates(grid, M, vel)
    front, _, rate_h = _eigen_calving_front(grid, M, edot, K)
    floating = m_floating_ice(M)
    nfl = np.zeros(M.shape)
    hsum = np.zeros(M.shape)
    for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        f = nb(floating, di, dj)
        nfl = nfl + f
        hsum = hsum + np.where(f, nb(H, di, dj), 0.0)
    H_average = np.where(nfl > 0, hsum / np.maximum(nfl, 1), hsum)
    calving_rate = rate_h * H_average / grid.dx
    hit = front & (calving_rate > 0.0)
    Href = np.where(hit, Href - calving_rate * dt, Href)
    gone = hit & (Href < 0.0)
    loss = np.where(gone, -Href, 0.0)
    Href = np.where(gone, 0.0, Href)
    loss = np.where(gone & (nfl > 0), loss / np.maximum(nfl, 1), loss)
    ln = [nb(loss, 1, 0), nb(loss, -1, 0), nb(loss, 0, 1), nb(loss, 0, -1)]
    cut = floating & ((ln[0] > 0.0) | (ln[1] > 0.0) | (ln[2] > 0.0) | (ln[3] > 0.0))
    total = ln[0] + ln[1] + ln[2] + ln[3]
    Href = np.where(cut, np.maximum(H - total, 0.0), Href)
    H = np.where(cut, 0.0, H)
    M = np.where(cut, MASK_ICE_FREE_OCEAN, M)
    M, H = remove_narrow_tongues(M, H)
    return M.astype(np.float64), Href, H


def eigen_calving_max_timestep(grid: Grid, mask, vel, K):
    """EigenCalving::max_timestep, PISMEigenCalving.cc:249-341: (dt, maximum rate, mean rate,
    number of cells calving) from the calving rates K e1 e2 (m/s) at the front cells, dt =
    max(1 / (max rate / dx + epsilon), 0.001 year)."""
    M = as_int(mask)
    edot = principal_strain_rates(grid, M, vel)
    _, calving, rate = _eigen_calving_front(grid, M, edot, K)
    count = float(np.count_nonzero(calving))
    rmax = max(0.0, float(np.max(rate[calving]))) if count > 0 else 0.0
    rmean = float(np.sum(rate[calving])) / count if count > 0 else 0.0
    dt_min = 0.001 * SECPERA
    epsilon = 0.001 / (grid.dx + grid.dy) / SECPERA
    dt = 1.0 / (rmax / grid.dx + epsilon)
    return max(dt, dt_min), rmax, rmean, count


def residual_rel(grid, cfg, inp, vel, reg, hardness, b):
    """||b - A(u) u||_2 / ||b||_2 with A built at the velocity itself (a nonlinear residual)."""
    nuH = compute_nuH(grid, cfg, inp, hardness, vel, reg)
    beta = beta_field(cfg, inp, vel)
    A = assemble_matrix(grid, cfg, inp, nuH, beta, check_diagonal=False)
    r = b.ravel() - A @ vel.ravel()
    return float(np.linalg.norm(r) / np.linalg.norm(b.ravel()))


def from_case(grid_desc, cfg_obj, fields) -> tuple[Grid, Config, Inputs]:
    """Adapt a (grid, config, fields) triple from any host builder (duck-typed)."""
    grid = Grid(grid_desc.Mx, grid_desc.My, grid_desc.Lx, grid_desc.Ly, grid_desc.x0,
                grid_desc.y0, grid_desc.periodicity,
                None if grid_desc.z is None else np.asarray(grid_desc.z, dtype=np.float64))
    kw = {}
    for name in Config.__dataclass_fields__:
        if hasattr(cfg_obj, name):
            kw[name] = getattr(cfg_obj, name)
    cfg = Config(**kw)
    inp = Inputs(**{k: (None if v is None else np.asarray(v, dtype=np.float64))
                    for k, v in fields.items() if k in Inputs.__dataclass_fields__})
    return grid, cfg, inp


# ---------------------------------------------------------------------------
# PETSc-like linear solve: GMRES(30) + block Jacobi / ILU(0) over the DMDA ranks
# ---------------------------------------------------------------------------
def compute_nprocs(Mx: int, My: int, size: int):
    """compute_nprocs, src/base/util/IceGrid.cc:395-430. Returns (Nx, Ny)."""
    Nx = int(0.5 + math.sqrt(float(Mx) * float(size) / float(My)))
    Ny = 0
    if Nx == 0:
        Nx = 1
    while Nx > 0:
        Ny = size // Nx
        if Nx * Ny == size:
            break
        Nx -= 1
    if Mx > My and Nx < Ny:
        Nx, Ny = Ny, Nx
    return Nx, Ny


def ownership_ranges(M: int, N: int):
    """ownership_ranges, IceGrid.cc:435-444."""
    return [M // N + ((M % N) > i) for i in range(N)]


def petsc_order(Mx: int, My: int, size: int):
    """Permutation from this module's unknown order to PETSc's rank-major DMDA order,
    and the rank block boundaries.  The DMDA is created as (M=My, N=Mx) with
    lx = procs_y, ly = procs_x (IceGrid.cc:800-823): ranks advance fastest in j."""
    Nx, Ny = compute_nprocs(Mx, My, size)
    px, py = ownership_ranges(Mx, Nx), ownership_ranges(My, Ny)
    xs = np.concatenate([[0], np.cumsum(px)])
    ys = np.concatenate([[0], np.cumsum(py)])
    perm = []
    starts = [0]
    for ry in range(Nx):          # PETSc "y" = PISM i
        for rx in range(Ny):      # PETSc "x" = PISM j
            I, J = np.meshgrid(np.arange(xs[ry], xs[ry + 1]), np.arange(ys[rx], ys[rx + 1]), indexing="ij")
            cells = (I * My + J).ravel()
            idx = np.stack([2 * cells, 2 * cells + 1], axis=1).ravel()
            perm.append(idx)
            starts.append(starts[-1] + idx.size)
    return np.concatenate(perm), np.array(starts, dtype=np.int32)


_KSP_LIB = None


def _ksp_lib():
    global _KSP_LIB
    if _KSP_LIB is None:
        import ctypes
        import os
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "libksp_cpu.so")
        lib = ctypes.CDLL(path)
        P = ctypes.POINTER
        lib.ksp_gmres_bjacobi_ilu0.restype = ctypes.c_int
        lib.ksp_gmres_bjacobi_ilu0.argtypes = [
            ctypes.c_int, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_double), ctypes.c_int,
            P(ctypes.c_int), P(ctypes.c_double), P(ctypes.c_double), ctypes.c_double, ctypes.c_double,
            ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, P(ctypes.c_int),
            P(ctypes.c_double), P(ctypes.c_double)]
        _KSP_LIB = lib
    return _KSP_LIB


def petsc_gmres_bjacobi(A, b, x0, Mx, My, nranks=1, rtol=1e-5, maxit=10000, restart=30,
                        nthreads=0, abstol=1e-50, dtol=1e5):
    """PETSc's default SSAFD linear solve restated (ksp_cpu.cc). Returns (x, its, reason)."""
    import ctypes
    perm, starts = petsc_order(Mx, My, nranks)
    Ap = A[perm][:, perm].tocsr()
    Ap.sort_indices()
    rp = np.ascontiguousarray(Ap.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(Ap.indices, dtype=np.int32)
    va = np.ascontiguousarray(Ap.data, dtype=np.float64)
    bp = np.ascontiguousarray(b[perm], dtype=np.float64)
    xp = np.ascontiguousarray(x0[perm], dtype=np.float64)
    its = ctypes.c_int(0)
    rn = ctypes.c_double(0)
    rn0 = ctypes.c_double(0)
    P = ctypes.POINTER
    lib = _ksp_lib()
    reason = lib.ksp_gmres_bjacobi_ilu0(
        Ap.shape[0], rp.ctypes.data_as(P(ctypes.c_int)), ci.ctypes.data_as(P(ctypes.c_int)),
        va.ctypes.data_as(P(ctypes.c_double)), len(starts) - 1, starts.ctypes.data_as(P(ctypes.c_int)),
        bp.ctypes.data_as(P(ctypes.c_double)), xp.ctypes.data_as(P(ctypes.c_double)), rtol, abstol, dtol,
        maxit, restart, nthreads, ctypes.byref(its), ctypes.byref(rn), ctypes.byref(rn0))
    x = np.empty_like(xp)
    x[perm] = xp
    return x, its.value, reason


def picard_native(grid: Grid, cfg: Config, inp: Inputs, hardness, b, vel0, reg, underrelax=1.0, nranks=1,
                  nthreads=0, ksp_rtol=1e-8, max_iterations=None, picard_rtol=None, ksp_maxit=10000, restart=30):
    """SSAFD::picard_manager on the host cores in native code (ssafd_cpu.cc): the same
    arithmetic as SSAFDOracle.picard_manager with linear="petsc" (nu*H, drag, the 18-column
    assembly in PETSc's rank-major order, GMRES(30) + block Jacobi / ILU(0) with one block
    per rank, under-relaxation, norms, stopping test).  No calving-front boundary condition,
    nu_bedrock or sub-grid grounding line (the benchmark sheet uses none of them).

    Returns (velocity, info) with info = {"status": 0 converged / 1 Picard limit / < 0 KSP
    reason, "picard_iterations", "nuH_norm", "nuH_norm_change", "ksp_iterations" [per
    iteration], "t_nuH", "t_assemble", "t_ksp" [seconds per iteration], "rel_change" [the
    relative nu*H change of each Picard test]}."""
    import ctypes
    if cfg.calving_front_stress_boundary_condition or cfg.nu_bedrock_set or cfg.sub_groundingline:
        raise ValueError("picard_native: CFBC, nu_bedrock and sub_groundingline are not restated natively")
    lib = _ksp_lib()
    if not hasattr(lib, "_picard_bound"):
        P = ctypes.POINTER
        D, I = ctypes.c_double, ctypes.c_int
        lib.ssafd_cpu_picard.restype = I
        lib.ssafd_cpu_picard.argtypes = [I, I, P(D), P(D), P(I), P(D), P(D), P(I), P(D), P(D), P(I), I, P(I), I, I,
                                         D, D, I, I, D, D, P(I), P(D), P(D), P(I), P(D), P(D), P(D), P(D)]
        lib._picard_bound = True
    Mx, My = grid.Mx, grid.My
    n_it = max_iterations if max_iterations is not None else cfg.max_iterations_ssafd
    rtol = picard_rtol if picard_rtol is not None else cfg.ssafd_relative_convergence
    par = np.array([grid.dx, grid.dy, cfg.ssa_Glen_exponent, cfg.ssa_enhancement_factor, schoof_reg(cfg),
                    cfg.min_thickness_strength_extension_ssa, cfg.constant_nu_strength_extension_ssa,
                    cfg.plastic_regularization, 1.0 if cfg.do_pseudo_plastic_till else 0.0, cfg.pseudo_plastic_q,
                    cfg.pseudo_plastic_uthreshold, cfg.sliding_scale_factor_reduces_tauc,
                    cfg.beta_ice_free_bedrock, cfg.scaling], dtype=np.float64)
    perm, starts = petsc_order(Mx, My, nranks)
    H = np.ascontiguousarray(inp.thickness, dtype=np.float64)
    mask = np.ascontiguousarray(as_int(inp.mask), dtype=np.int32)
    tauc = np.ascontiguousarray(inp.tauc, dtype=np.float64)
    hard = np.ascontiguousarray(hardness, dtype=np.float64)
    bc = None
    if inp.bc_mask is not None and inp.bc_values is not None:
        bc = np.ascontiguousarray(as_int(inp.bc_mask) == 1, dtype=np.int32)
    bb = np.ascontiguousarray(b, dtype=np.float64).ravel()
    vel = np.ascontiguousarray(np.array(vel0, dtype=np.float64).reshape(Mx, My, 2))
    perm = np.ascontiguousarray(perm, dtype=np.int32)
    starts = np.ascontiguousarray(starts, dtype=np.int32)
    its = np.zeros(n_it, dtype=np.int32)
    t_nuH, t_asm, t_ksp, relc = np.zeros(n_it), np.zeros(n_it), np.zeros(n_it), np.zeros(n_it)
    npic = ctypes.c_int(0)
    norm, change = ctypes.c_double(0), ctypes.c_double(0)
    P = ctypes.POINTER

    def dp(a):
        return a.ctypes.data_as(P(ctypes.c_double))

    def ip(a):
        return a.ctypes.data_as(P(ctypes.c_int)) if a is not None else None

    st = lib.ssafd_cpu_picard(Mx, My, dp(par), dp(H), ip(mask), dp(tauc), dp(hard), ip(bc), dp(bb), dp(vel),
                              ip(perm), len(starts) - 1, ip(starts), nthreads, n_it, rtol, ksp_rtol, ksp_maxit,
                              restart, reg, underrelax, ctypes.byref(npic), ctypes.byref(norm),
                              ctypes.byref(change), ip(its), dp(t_nuH), dp(t_asm), dp(t_ksp), dp(relc))
    k = npic.value
    m = k if st >= 0 else k + 1
    return vel, {"status": st, "picard_iterations": k, "nuH_norm": norm.value, "nuH_norm_change": change.value,
                 "ksp_iterations": its[:m].tolist(), "t_nuH": t_nuH[:k].tolist(), "t_assemble": t_asm[:k].tolist(),
                 "t_ksp": t_ksp[:k].tolist(), "rel_change": relc[:k].tolist()}
