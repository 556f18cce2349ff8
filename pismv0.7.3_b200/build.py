"""Build recipe of the B200 SSA solver: nvcc for sm_100a, in-tree output.

    python pismv0.7.3_b200/build.py        (or build() from __graft_entry__)

Produces lib/libpism_ssa_gpu.so (the C-ABI of include/pism_ssa_gpu.h) and
lib/ssa_test_gpu (the C++ verification driver, a counterpart of the reference's
ssa_testi / ssa_testj / ssa_test_cfbc executables).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
CU_SOURCES = ["ssa_kernels.cu", "ssa_mg.cu", "ssa_mixed.cu", "ssa_line.cu", "ssa_control.cu", "ssa_capi.cu", "ssa_noalloc.cu", "unet.cu",
              "ssa_column.cu", "ssa_transport.cu", "ssa_calving.cu",
              "ssa_fem.cu"]


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    so = os.path.join(LIB, "libpism_ssa_gpu.so")
    inc = os.path.join(REPO, "include")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(inc, f) for f in os.listdir(inc)]
    if force or _newer(so, deps):
        cmd = ["nvcc", *NVCC_FLAGS, "-I", inc, "-shared", "-o", so, *[os.path.join(CSRC, f) for f in CU_SOURCES]]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    drv = os.path.join(LIB, "ssa_test_gpu")
    drv_src = [os.path.join(CSRC, "host", f) for f in ("SSAFD_GPU.cc", "ssa_test_gpu.cc")]
    if all(os.path.exists(s) for s in drv_src) and (force or _newer(drv, drv_src + [so])):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(REPO, "include"), "-I",
               os.path.join(CSRC, "host"), *drv_src, "-o", drv, "-L", LIB, "-lpism_ssa_gpu",
               "-Wl,-rpath,$ORIGIN", "-lm"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return so


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
