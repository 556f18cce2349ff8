"""The C-ABI boundary without a GPU: exports, struct layout, defaults, host-side logic."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from pism_b200 import _capi, build as B
from pism_b200.config import CConfig, CGrid, CInputs, CMember, CStats, SSAConfig, GridDesc

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "pism_ssa_gpu.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|void|const char \*)\s*(pism_gpu_ssa(?:fem)?_\w+)\s*\(", txt, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return _capi.load()


def test_library_exports_every_declared_symbol(lib):
    decl = declared_functions()
    assert len(decl) >= 15
    assert sorted(_capi.EXPORTS) == decl
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (pism_gpu_ssa(?:fem)?_\w+)", out))
    missing = [d for d in decl if d not in exported]
    assert not missing, missing
    for d in decl:
        assert hasattr(lib, d)


def test_unet_library_exports_every_declared_symbol(lib):
    txt = open(os.path.join(REPO, "include", "pism_unet_gpu.h")).read()
    decl = sorted(set(re.findall(r"^(?:int|const char \*|long long)\s*(pism_gpu_\w+)\s*\(", txt, flags=re.M)))
    assert sorted(_capi.UNET_EXPORTS) == decl
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (pism_gpu_\w+)", out))
    assert not [d for d in decl if d not in exported]


def test_unet_param_count_matches_the_oracle(lib):
    from oracle import unet_oracle as U
    assert lib.pism_gpu_unet_param_count() == U.param_count()


def test_unet_rejects_bad_shapes_without_touching_cuda(lib):
    h = C.c_void_p()
    for args in ((0, 0, 16, 16), (0, 1, 12, 16), (0, 1, 16, 4), (0, 1, 0, 16)):
        assert lib.pism_gpu_unet_create(*args, C.byref(h)) == _capi.EINVAL


def _c_layout():
    """sizeof / offsetof of the C structs, compiled from the header with gcc."""
    src = r'''
#include <stddef.h>
#include <stdio.h>
#include "pism_ssa_gpu.h"
#define F(T, m) printf(#T " " #m " %zu\n", offsetof(T, m));
int main(void) {
  printf("pism_gpu_ssa_config size %zu\n", sizeof(pism_gpu_ssa_config));
  printf("pism_gpu_grid size %zu\n", sizeof(pism_gpu_grid));
  printf("pism_gpu_ssa_inputs size %zu\n", sizeof(pism_gpu_ssa_inputs));
  printf("pism_gpu_ssa_stats size %zu\n", sizeof(pism_gpu_ssa_stats));
  printf("pism_gpu_ssa_member size %zu\n", sizeof(pism_gpu_ssa_member));
  F(pism_gpu_ssa_member, ice_softness) F(pism_gpu_ssa_member, velocity)
  F(pism_gpu_ssa_config, ksp_rtol) F(pism_gpu_ssa_config, verbosity) F(pism_gpu_ssa_config, mg_omega)
  F(pism_gpu_ssa_config, flow_law) F(pism_gpu_ssa_config, brutal_sliding_scale)
  F(pism_gpu_grid, z) F(pism_gpu_ssa_inputs, fracture_density) F(pism_gpu_ssa_stats, kernel_launches)
  return 0;
}
'''
    d = os.path.join(REPO, "oracle", "_build")
    os.makedirs(d, exist_ok=True)
    cpath, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
    open(cpath, "w").write(src)
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), cpath, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    return {tuple(line.split()[:2]): int(line.split()[2]) for line in out.strip().splitlines()}


def test_ctypes_structs_match_the_header():
    lay = _c_layout()
    assert lay[("pism_gpu_ssa_config", "size")] == C.sizeof(CConfig)
    assert lay[("pism_gpu_grid", "size")] == C.sizeof(CGrid)
    assert lay[("pism_gpu_ssa_inputs", "size")] == C.sizeof(CInputs)
    assert lay[("pism_gpu_ssa_stats", "size")] == C.sizeof(CStats)
    assert lay[("pism_gpu_ssa_member", "size")] == C.sizeof(CMember)
    for (struct, member), off in lay.items():
        if member == "size":
            continue
        cls = {"pism_gpu_ssa_config": CConfig, "pism_gpu_grid": CGrid, "pism_gpu_ssa_inputs": CInputs,
               "pism_gpu_ssa_stats": CStats, "pism_gpu_ssa_member": CMember}[struct]
        assert getattr(cls, member).offset == off, (struct, member)


def test_config_defaults_agree(lib):
    """pism_gpu_ssa_config_defaults (C) and SSAConfig (Python) carry the same pism_config.cdl values."""
    c = CConfig()
    assert lib.pism_gpu_ssa_config_defaults(C.byref(c)) == 0
    py = SSAConfig().to_c()
    for name, _ in CConfig._fields_:
        a, b = getattr(c, name), getattr(py, name)
        if name in ("flow_law",):
            assert a == b
        elif isinstance(a, float):
            assert a == pytest.approx(b, rel=1e-15), name
        else:
            assert a == b, name


def test_create_rejects_bad_grids_without_touching_cuda(lib):
    cfg = CConfig()
    lib.pism_gpu_ssa_config_defaults(C.byref(cfg))
    h = C.c_void_p()
    for Mx, My, dx in ((2, 10, 1.0), (10, 2, 1.0), (10, 10, 0.0)):
        g = CGrid(Mx, My, dx, 1.0, 0, 0, None)
        assert lib.pism_gpu_ssa_create(C.byref(g), C.byref(cfg), 0, C.byref(h)) == _capi.EINVAL
    assert lib.pism_gpu_ssa_create(None, C.byref(cfg), 0, C.byref(h)) == _capi.EINVAL


def test_gmres_settings_are_checked_before_device_work(lib):
    """ksp_type GMRES: restart in [1, 30]; the mixed-precision inner solve stays BiCGStab."""
    g, _z = GridDesc(16, 16, 1e5, 1e5).to_c()
    h = C.c_void_p()
    for kw in ({"ksp_type": "gmres", "gmres_restart": 0}, {"ksp_type": "gmres", "gmres_restart": 31},
               {"ksp_type": "gmres", "precision": "mixed", "pc_type": "mg"}, {"graphs": 4}, {"graphs": -1}, {"mg_post_blocks_per_sm": 5}):
        cfg = SSAConfig(**kw).to_c()
        assert lib.pism_gpu_ssa_create(C.byref(g), C.byref(cfg), 0, C.byref(h)) == _capi.EINVAL, kw


def test_noalloc_rejects_before_any_device_work(lib):
    """Size and argument checks of the allocation-free entry point happen on the host."""
    cfg = SSAConfig().to_c()
    g, _z = GridDesc(4096, 4096, 1e6, 1e6).to_c()
    dummy = C.c_void_p(16)
    rc = lib.pism_gpu_ssa_nuH_noalloc(C.byref(g), C.byref(cfg), dummy, dummy, dummy, dummy, dummy, None, 0.0, 1.0,
                                      dummy, dummy, dummy, None)
    assert rc == _capi.ETOOLARGE
    rc = lib.pism_gpu_ssa_nuH_noalloc(C.byref(g), C.byref(cfg), None, dummy, dummy, dummy, dummy, None, 0.0, 1.0,
                                      dummy, dummy, dummy, None)
    assert rc == _capi.EINVAL


def test_host_driver_is_built(lib):
    exe = os.path.join(REPO, "pismv0.7.3_b200", "lib", "ssa_test_gpu")
    assert os.access(exe, os.X_OK)
    r = subprocess.run([exe, "-test", "X"], capture_output=True, text=True)
    assert r.returncode == 2 and "unknown test" in r.stderr


def test_host_driver_rejects_short_parameter_files(lib, tmp_path):
    """-learned reads pism_gpu_unet_param_count() floats; a short or missing file is an
    error before any device work."""
    exe = os.path.join(REPO, "pismv0.7.3_b200", "lib", "ssa_test_gpu")
    short = tmp_path / "short.f32"
    np.zeros(100, np.float32).tofile(short)
    for path in (str(short), str(tmp_path / "missing.f32")):
        r = subprocess.run([exe, "-test", "I", "-My", "61", "-learned", path], capture_output=True, text=True)
        assert r.returncode == 2 and "cannot load the network parameters" in r.stderr


def test_grid_coordinates_match_icegrid():
    """GridDesc follows IceGrid::compute_horizontal_coordinates (IceGrid.cc:550-610)."""
    g = GridDesc(5, 7, 60e3, 120e3, periodicity=2)
    x, y = g.x_coords(), g.y_coords()
    np.testing.assert_allclose(x, [-60e3, -30e3, 0, 30e3, 60e3])
    dy = 240e3 / 7
    assert g.dy == pytest.approx(dy)
    assert y[0] == pytest.approx(-120e3 + 0.5 * dy) and y[-1] == pytest.approx(120e3 - 0.5 * dy)


def _header_enum(prefix):
    text = open(os.path.join(REPO, "include", "pism_ssa_gpu.h")).read()
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"\b(" + prefix + r"\w+)\s*=\s*(\d+)", text)}


def test_option_tables_match_the_header():
    """The Python option names map to the header's enum values."""
    from pism_b200 import config as Cfg
    pc = _header_enum("PISM_PC_")
    assert Cfg.PC_TYPES == {"bjacobi": pc["PISM_PC_BLOCK_JACOBI"], "mg": pc["PISM_PC_MULTIGRID"],
                            "line": pc["PISM_PC_LINE"]}
    ksp = _header_enum("PISM_KSP_")
    assert Cfg.KSP_TYPES == {"bicgstab": ksp["PISM_KSP_BICGSTAB"], "gmres": ksp["PISM_KSP_GMRES"]}
    prec = _header_enum("PISM_PRECISION_")
    assert Cfg.PRECISIONS == {"fp64": prec["PISM_PRECISION_FP64"], "mixed": prec["PISM_PRECISION_MIXED"]}
    law = _header_enum("PISM_FLOW_LAW_")
    assert Cfg.FLOW_LAWS == {"isothermal_glen": law["PISM_FLOW_LAW_ISOTHERMAL_GLEN"], "pb": law["PISM_FLOW_LAW_PB"],
                             "gpbld": law["PISM_FLOW_LAW_GPBLD"], "arr": law["PISM_FLOW_LAW_ARR"],
                             "arrwarm": law["PISM_FLOW_LAW_ARRWARM"], "hooke": law["PISM_FLOW_LAW_HOOKE"]}
