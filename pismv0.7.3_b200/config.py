"""SSA configuration and grid description, mirrored onto the C-ABI structs.

``SSAConfig`` carries the pism_config.cdl parameters that the SSAFD path reads
(names unchanged; defaults from src/pism_config.cdl, converted to SI as PISM's
Config::get_double(name, "m/s") would).  ``GridDesc`` follows
IceGrid::compute_horizontal_spacing / compute_coordinates (IceGrid.cc:540-610).
Both convert to the ctypes structs declared in include/pism_ssa_gpu.h.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields, replace

import numpy as np

SECPERA = 31556925.9747  # UDUNITS-2 year, used by PISM's m/year <-> m/s conversions

X_PERIODIC = 1
Y_PERIODIC = 2
XY_PERIODIC = 3

FLOW_LAWS = {"isothermal_glen": 0, "pb": 1, "gpbld": 2, "arr": 3, "arrwarm": 4, "hooke": 5}
KSP_TYPES = {"bicgstab": 0, "gmres": 1}
PC_TYPES = {"bjacobi": 0, "mg": 1, "line": 2}
PRECISIONS = {"fp64": 0, "mixed": 1}


@dataclass
class SSAConfig:
    ice_density: float = 910.0
    sea_water_density: float = 1028.0
    standard_gravity: float = 9.81
    sea_level: float = 0.0
    epsilon_ssa: float = 1.0e13
    ssafd_relative_convergence: float = 1.0e-4
    max_iterations_ssafd: int = 300
    ssafd_nuH_iter_failure_underrelaxation: float = 0.8
    min_thickness_strength_extension_ssa: float = 50.0
    constant_nu_strength_extension_ssa: float = 9.48680701906572e14
    plastic_regularization: float = 0.01 / SECPERA
    do_pseudo_plastic_till: bool = False
    pseudo_plastic_q: float = 0.25
    pseudo_plastic_uthreshold: float = 100.0 / SECPERA
    sliding_scale_factor_reduces_tauc: float = -1.0
    beta_ice_free_bedrock: float = 1.8e9
    calving_front_stress_boundary_condition: bool = False
    ssa_dirichlet_bc: bool = False
    sub_groundingline: bool = False
    nu_bedrock_set: bool = False
    nu_bedrock: float = 5.0e15
    surface_gradient_method: str = "haseloff"
    compute_surf_grad_inward_ssa: bool = False
    flow_law: str = "gpbld"
    ssa_Glen_exponent: float = 3.0
    ssa_enhancement_factor: float = 1.0
    ice_softness: float = 3.1689e-24
    Schoof_regularizing_length: float = 1000.0e3
    Schoof_regularizing_velocity: float = 1.0 / SECPERA
    Paterson_Budd_A_cold: float = 3.61e-13
    Paterson_Budd_A_warm: float = 1.73e3
    Paterson_Budd_Q_cold: float = 6.0e4
    Paterson_Budd_Q_warm: float = 13.9e4
    Paterson_Budd_critical_temperature: float = 263.15
    ideal_gas_constant: float = 8.31441
    gpbld_water_frac_coeff: float = 181.25
    gpbld_water_frac_observed_limit: float = 0.01
    Hooke_A: float = 4.42165e-9
    Hooke_Q: float = 7.88e4
    Hooke_C: float = 0.16612
    Hooke_k: float = 1.17
    Hooke_Tr: float = 273.39
    beta_CC: float = 7.9e-8
    ice_specific_heat_capacity: float = 2009.0
    water_latent_heat_fusion: float = 3.34e5
    surface_pressure: float = 0.0
    water_melting_point_temperature: float = 273.15
    enthalpy_converter_reference_temperature: float = 223.15
    do_fracture_density: bool = False
    fracture_density_softening_lower_limit: float = 1.0
    brutal_sliding: bool = False
    brutal_sliding_scale: float = 1.0
    # linear solver (the reference's -ssafd_ksp_* options; PETSc defaults)
    ksp_type: str = "bicgstab"
    pc_type: str = "bjacobi"
    ksp_rtol: float = 1.0e-5
    ksp_max_it: int = 10000
    gmres_restart: int = 30
    precision: str = "fp64"
    mixed_inner_rtol: float = 1.0e-3
    mg_omega: float = 0.9
    mg_correction: float = 1.2
    ksp_rtol_adaptive: bool = False
    ksp_rtol_max: float = 1.0e-2
    ksp_rtol_factor: float = 1.0e-2
    graphs: int = 2
    verbosity: int = 0
    mg_post_blocks_per_sm: int = 0
    mg_rebuild_rtol: float = 0.0
    mg_small_kernel: int = 0
    mixed_apply_kernel: int = 2
    # geometry helpers (not part of the C struct)
    mask_icefree_thickness_standard: float = 0.01
    mask_is_floating_thickness_standard: float = 1.0

    def copy(self, **kw) -> "SSAConfig":
        return replace(self, **kw)

    def to_c(self) -> "CConfig":
        c = CConfig()
        for name, _ in CConfig._fields_:
            if name == "surface_gradient_eta":
                val = 1 if self.surface_gradient_method == "eta" else 0
            elif name == "flow_law":
                val = FLOW_LAWS[self.flow_law]
            elif name == "ksp_type":
                val = KSP_TYPES[self.ksp_type]
            elif name == "pc_type":
                val = PC_TYPES[self.pc_type]
            elif name == "precision":
                val = PRECISIONS[self.precision]
            else:
                val = getattr(self, name)
            setattr(c, name, int(val) if isinstance(val, bool) else val)
        return c


_D, _I = C.c_double, C.c_int


class CConfig(C.Structure):
    """ctypes image of pism_gpu_ssa_config (include/pism_ssa_gpu.h)."""
    _fields_ = [
        ("ice_density", _D), ("sea_water_density", _D), ("standard_gravity", _D), ("sea_level", _D),
        ("epsilon_ssa", _D), ("ssafd_relative_convergence", _D), ("max_iterations_ssafd", _I),
        ("ssafd_nuH_iter_failure_underrelaxation", _D), ("min_thickness_strength_extension_ssa", _D),
        ("constant_nu_strength_extension_ssa", _D), ("plastic_regularization", _D),
        ("do_pseudo_plastic_till", _I), ("pseudo_plastic_q", _D), ("pseudo_plastic_uthreshold", _D),
        ("sliding_scale_factor_reduces_tauc", _D), ("beta_ice_free_bedrock", _D),
        ("calving_front_stress_boundary_condition", _I), ("ssa_dirichlet_bc", _I),
        ("sub_groundingline", _I), ("nu_bedrock_set", _I), ("nu_bedrock", _D),
        ("surface_gradient_eta", _I), ("compute_surf_grad_inward_ssa", _I), ("flow_law", _I),
        ("ssa_Glen_exponent", _D), ("ssa_enhancement_factor", _D), ("ice_softness", _D),
        ("Schoof_regularizing_length", _D), ("Schoof_regularizing_velocity", _D),
        ("Paterson_Budd_A_cold", _D), ("Paterson_Budd_A_warm", _D), ("Paterson_Budd_Q_cold", _D),
        ("Paterson_Budd_Q_warm", _D), ("Paterson_Budd_critical_temperature", _D),
        ("ideal_gas_constant", _D), ("gpbld_water_frac_coeff", _D), ("gpbld_water_frac_observed_limit", _D),
        ("Hooke_A", _D), ("Hooke_Q", _D), ("Hooke_C", _D), ("Hooke_k", _D), ("Hooke_Tr", _D),
        ("beta_CC", _D), ("ice_specific_heat_capacity", _D), ("water_latent_heat_fusion", _D),
        ("surface_pressure", _D), ("water_melting_point_temperature", _D),
        ("enthalpy_converter_reference_temperature", _D), ("do_fracture_density", _I),
        ("fracture_density_softening_lower_limit", _D), ("brutal_sliding", _I),
        ("brutal_sliding_scale", _D), ("ksp_type", _I), ("pc_type", _I), ("ksp_rtol", _D),
        ("ksp_max_it", _I), ("gmres_restart", _I), ("precision", _I), ("mixed_inner_rtol", _D),
        ("mg_omega", _D), ("mg_correction", _D), ("ksp_rtol_adaptive", _I), ("ksp_rtol_max", _D),
        ("ksp_rtol_factor", _D), ("graphs", _I), ("verbosity", _I), ("mg_post_blocks_per_sm", _I),
        ("mg_rebuild_rtol", _D), ("mg_small_kernel", _I), ("mixed_apply_kernel", _I),
    ]


class CGrid(C.Structure):
    _fields_ = [("Mx", _I), ("My", _I), ("dx", _D), ("dy", _D), ("periodicity", _I),
                ("Mz", _I), ("z", C.POINTER(_D))]


class CInputs(C.Structure):
    _fields_ = [("where", _I)] + [(n, C.POINTER(_D)) for n in (
        "thickness", "surface", "bed", "mask", "tauc", "bc_mask", "bc_values", "melange",
        "gl_mask", "enthalpy", "hardness_stag", "fracture_density")]


class CMember(C.Structure):
    _fields_ = [("inputs", CInputs), ("ice_softness", _D), ("velocity", C.POINTER(_D))]


class CStats(C.Structure):
    _fields_ = [("status", _I), ("converged", _I), ("strategy", _I), ("picard_iterations", _I),
                ("ksp_iterations", _I), ("ksp_failures", _I), ("refinement_steps", _I),
                ("nuH_norm", _D), ("nuH_norm_change", _D), ("final_linear_residual", _D),
                ("solve_ms", _D), ("kernel_ms", _D), ("kernel_launches", C.c_longlong), ("mg_rebuilds", _I)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class CFemOptions(C.Structure):
    """pism_gpu_ssafem_options"""
    _fields_ = [("snes_rtol", _D), ("snes_stol", _D), ("snes_max_it", _I), ("ksp_rtol", _D), ("ksp_max_it", _I),
                ("dirichlet_scale", _D), ("icefree_thickness", _D), ("is_floating_thickness", _D)]


class CFemStats(C.Structure):
    """pism_gpu_ssafem_stats"""
    _fields_ = [("converged", _I), ("newton_iterations", _I), ("ksp_iterations", _I), ("fnorm0", _D),
                ("fnorm", _D)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


@dataclass
class GridDesc:
    Mx: int
    My: int
    Lx: float
    Ly: float
    x0: float = 0.0
    y0: float = 0.0
    periodicity: int = 0
    z: np.ndarray | None = None

    @classmethod
    def shallow(cls, Mx, My, Lx, Ly, periodicity=0, x0=0.0, y0=0.0):
        """IceGrid::Shallow: a grid with 3 vertical levels on [0, 1000] (IceGrid.cc:148-176)."""
        return cls(Mx, My, Lx, Ly, x0, y0, periodicity, np.array([0.0, 500.0, 1000.0]))

    @property
    def dx(self) -> float:
        return 2.0 * self.Lx / (self.Mx if self.periodicity & X_PERIODIC else self.Mx - 1)

    @property
    def dy(self) -> float:
        return 2.0 * self.Ly / (self.My if self.periodicity & Y_PERIODIC else self.My - 1)

    @staticmethod
    def _coords(M, delta, vmin, vmax, periodic):
        if periodic:
            r = vmin + (np.arange(M) + 0.5) * delta
            r[M - 1] = vmax - 0.5 * delta
        else:
            r = vmin + np.arange(M) * delta
            r[M - 1] = vmax
        return r

    def x_coords(self):
        return self._coords(self.Mx, self.dx, self.x0 - self.Lx, self.x0 + self.Lx,
                            bool(self.periodicity & X_PERIODIC))

    def y_coords(self):
        return self._coords(self.My, self.dy, self.y0 - self.Ly, self.y0 + self.Ly,
                            bool(self.periodicity & Y_PERIODIC))

    def to_c(self) -> tuple[CGrid, object]:
        z = np.ascontiguousarray(self.z if self.z is not None else np.zeros(0), dtype=np.float64)
        g = CGrid(self.Mx, self.My, self.dx, self.dy, self.periodicity, len(z),
                  z.ctypes.data_as(C.POINTER(_D)) if len(z) else None)
        return g, z  # keep z alive while g is in use
