"""B200-native finite-difference SSA (SSAFD) stress-balance solver for PISM v0.7.3.

The solver itself is ``libpism_ssa_gpu.so`` (CUDA, sm_100a) behind the C-ABI of
``include/pism_ssa_gpu.h``; this package holds its build recipe, the ctypes
binding, the host-side mirror of PISM's SSA interface (``ssa.SSAFD``), the
verification test cases I/J/V and the seeded synthetic benchmark geometries.
"""
from .config import SSAConfig, GridDesc, SECPERA, X_PERIODIC, Y_PERIODIC, XY_PERIODIC  # noqa: F401
from . import verification, synthetic  # noqa: F401


def __getattr__(name):
    if name in ("SSAFD", "SSAFD_GPUFactory", "KSPFailure", "PicardFailure", "SSAError", "ZeroDiagonal"):
        from . import ssa
        return getattr(ssa, name)
    raise AttributeError(name)
