"""ctypes binding of include/pism_ssa_gpu.h (libpism_ssa_gpu.so, built in-tree by build.py).

There is no fallback: if the shared library is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .config import CConfig, CFemOptions, CFemStats, CGrid, CInputs, CMember, CStats

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpism_ssa_gpu.so")

# status codes (PISM_GPU_SSA_*)
OK, EINVAL, ECUDA, ENOMEM, EKSP, EPICARD, EZERODIAG, ENAN, ESTATE, ETOOLARGE = range(10)
NOALLOC_MAX_CELLS = 2048 * 2048
# fields (PISM_FIELD_*)
FIELD_VELOCITY, FIELD_TAUD, FIELD_RHS, FIELD_HARDNESS, FIELD_NUH, FIELD_BETA, FIELD_BFRICT = range(7)
MEM_HOST, MEM_DEVICE = 0, 1

# every symbol include/pism_ssa_gpu.h declares
EXPORTS = [
    "pism_gpu_ssa_config_defaults", "pism_gpu_ssa_create", "pism_gpu_ssa_destroy", "pism_gpu_ssa_last_error",
    "pism_gpu_ssa_set_stream", "pism_gpu_ssa_set_config", "pism_gpu_ssa_set_inputs",
    "pism_gpu_ssa_set_initial_guess", "pism_gpu_ssa_solve", "pism_gpu_ssa_get_field",
    "pism_gpu_ssa_assemble_rhs", "pism_gpu_ssa_compute_hardness", "pism_gpu_ssa_compute_nuH",
    "pism_gpu_ssa_apply", "pism_gpu_ssa_apply_preconditioner", "pism_gpu_ssa_linear_solve",
    "pism_gpu_ssa_linear_solve_rhs", "pism_gpu_ssa_stress_balance_3d", "pism_gpu_ssa_mass_continuity_step",
    "pism_gpu_ssa_strain_rates", "pism_gpu_ssa_eigen_calving", "pism_gpu_ssa_eigen_calving_max_timestep",
    "pism_gpu_ssafem_options_defaults", "pism_gpu_ssafem_solve",
    "pism_gpu_ssa_nuH_noalloc", "pism_gpu_ssa_solve_batch",
]
# every symbol include/pism_unet_gpu.h declares
UNET_EXPORTS = [
    "pism_gpu_unet_param_count", "pism_gpu_unet_create", "pism_gpu_unet_destroy", "pism_gpu_unet_last_error",
    "pism_gpu_unet_set_stream", "pism_gpu_unet_set_params", "pism_gpu_unet_get_params", "pism_gpu_unet_forward",
    "pism_gpu_unet_backward", "pism_gpu_unet_adam", "pism_gpu_ssa_learned_features", "pism_gpu_ssa_learned_guess",
    "pism_gpu_ssa_set_learned_pc", "pism_gpu_ssa_learned_pc_input",
]

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m build` from the package "
                          "(pismv0.7.3_b200/build.py) — there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    P, I, D, V = C.POINTER, C.c_int, C.c_double, C.c_void_p
    sig = {
        "pism_gpu_ssa_config_defaults": (I, [P(CConfig)]),
        "pism_gpu_ssa_create": (I, [P(CGrid), P(CConfig), I, P(V)]),
        "pism_gpu_ssa_destroy": (I, [V]),
        "pism_gpu_ssa_last_error": (C.c_char_p, [V]),
        "pism_gpu_ssa_set_stream": (I, [V, V]),
        "pism_gpu_ssa_set_config": (I, [V, P(CConfig)]),
        "pism_gpu_ssa_set_inputs": (I, [V, P(CInputs)]),
        "pism_gpu_ssa_set_initial_guess": (I, [V, P(D), I]),
        "pism_gpu_ssa_solve": (I, [V, P(D), I, P(CStats)]),
        "pism_gpu_ssa_get_field": (I, [V, I, P(D), I]),
        "pism_gpu_ssa_assemble_rhs": (I, [V]),
        "pism_gpu_ssa_compute_hardness": (I, [V]),
        "pism_gpu_ssa_compute_nuH": (I, [V, D]),
        "pism_gpu_ssa_apply": (I, [V, V, V]),
        "pism_gpu_ssa_apply_preconditioner": (I, [V, V, V]),
        "pism_gpu_ssa_linear_solve": (I, [V, V, P(I), P(D)]),
        "pism_gpu_ssa_linear_solve_rhs": (I, [V, V, V, P(I), P(D)]),
        "pism_gpu_ssa_stress_balance_3d": (I, [V, P(D), P(D), P(D), P(D), P(D), I]),
        "pism_gpu_ssa_mass_continuity_step": (I, [V, D, P(D), P(D), P(D), D, D, P(D), P(D), P(D), P(D), P(D), I]),
        "pism_gpu_ssa_strain_rates": (I, [V, P(D), P(D), P(D), I]),
        "pism_gpu_ssa_eigen_calving": (I, [V, D, D, P(D), P(D), P(D), I]),
        "pism_gpu_ssa_eigen_calving_max_timestep": (I, [V, D, P(D), P(D), I]),
        "pism_gpu_ssafem_options_defaults": (None, [P(CFemOptions)]),
        "pism_gpu_ssafem_solve": (I, [V, P(CFemOptions), P(CFemStats)]),
        "pism_gpu_ssa_nuH_noalloc": (I, [P(CGrid), P(CConfig), V, V, V, V, V, V, D, D, V, V, V, V]),
        "pism_gpu_ssa_solve_batch": (I, [V, V, I, I, P(CMember), P(CStats)]),
        "pism_gpu_unet_param_count": (C.c_longlong, []),
        "pism_gpu_unet_create": (I, [I, I, I, I, P(V)]),
        "pism_gpu_unet_destroy": (I, [V]),
        "pism_gpu_unet_last_error": (C.c_char_p, [V]),
        "pism_gpu_unet_set_stream": (I, [V, V]),
        "pism_gpu_unet_set_params": (I, [V, V, I]),
        "pism_gpu_unet_get_params": (I, [V, V, I]),
        "pism_gpu_unet_forward": (I, [V, V, I, I, I, V]),
        "pism_gpu_unet_backward": (I, [V, V, V, P(C.c_float), V]),
        "pism_gpu_unet_adam": (I, [V, C.c_float, C.c_float, C.c_float, C.c_float]),
        "pism_gpu_ssa_learned_features": (I, [V, I, V, I, I]),
        "pism_gpu_ssa_learned_guess": (I, [V, V, I]),
        "pism_gpu_ssa_set_learned_pc": (I, [V, V, I]),
        "pism_gpu_ssa_learned_pc_input": (I, [V, I, V, V, I, I, V]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
