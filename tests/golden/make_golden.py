"""Generate tests/golden/reference_goldens.json from the reference tree.

Run where the reference checkout is present, naming its root (or setting
PISM_REFERENCE_ROOT):

    python tests/golden/make_golden.py REFERENCE_ROOT

What it records (nothing here is run at test time; the JSON is committed):

* the verification-test error tables that the reference's regression scripts
  diff against (test/regression/ssa/ssa_testi_fd.sh, ssa_testj_fd.sh,
  ssa_test_cfbc.sh; the SSAFEM scripts ssa_testi_fem.sh, ssa_testj_fem.sh,
  ssafem_test_linear.sh, ssafem_test_plug.sh), parsed from the scripts' heredocs, with
  the command-line options each was produced with;
* the test-I error table of doc/verif/I_userman_may2012.nc (FD solver, Mx = 5);
* the flow-law tables of test/regression/test_20.sh (gpbld), test_21.sh (pb),
  test_24.sh (hooke) and test_26.sh (arr);
* exactI / exactJ values at a fixed set of points, computed by the reference's own
  src/verif/tests/exactTestsIJ.c compiled in place (oracle/Makefile -> oracle/_ref).
"""
from __future__ import annotations

import ctypes
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def parse_error_tables(path):
    """Rows printed by SSATestCase::report between 'velocity  :' and 'NUM ERRORS DONE'."""
    txt = open(path).read()
    body = txt.split("<<END-OF-OUTPUT", 1)[1].split("END-OF-OUTPUT", 1)[0]
    rows = []
    lines = body.strip().splitlines()
    for k, line in enumerate(lines):
        if line.startswith("velocity  :"):
            vals = [float(v) for v in lines[k + 1].split()]
            rows.append(dict(zip(["maxvector", "prcntavvec", "maxu", "maxv", "avu", "avv"], vals)))
    return rows


def parse_flow_table(path):
    txt = open(path).read()
    body = txt.split("<<END-OF-OUTPUT", 1)[1].split("END-OF-OUTPUT", 1)[0]
    name = re.search(r'flow law:\s+"([^"]+)"', body).group(1)
    pressure = float(re.search(r"pressure = ([0-9.e+-]+) Pa", body).group(1))
    rows = []
    for line in body.splitlines():
        m = re.match(r"\s+([0-9.e+-]+)\s+([0-9.]+)\s+([0-9.]+) = ([0-9.e+-]+)", line)
        if m:
            rows.append([float(g) for g in m.groups()])
    return {"name": name, "pressure": pressure, "rows": rows}


def main(ref):
    out = {"source": "generated by tests/golden/make_golden.py from the PISM v0.7.3 reference tree"}
    ssa = os.path.join(ref, "test/regression/ssa")
    out["test_i_fd"] = {
        "script": "test/regression/ssa/ssa_testi_fd.sh:26-45",
        "options": {"Mx": 5, "ssa_rtol": 5e-7, "ksp_rtol": 1e-12, "mpi_ranks": 2},
        "cases": [dict(My=My, **row) for My, row in zip((61, 121), parse_error_tables(
            os.path.join(ssa, "ssa_testi_fd.sh")))],
    }
    out["test_j_fd"] = {
        "script": "test/regression/ssa/ssa_testj_fd.sh:25-44",
        "options": {"ssa_rtol": 1e-4, "ksp": "PETSc default gmres(30)+bjacobi/ilu(0), rtol 1e-5",
                    "mpi_ranks": 2},
        "cases": [dict(Mx=M, My=M, **row) for M, row in zip((61, 121), parse_error_tables(
            os.path.join(ssa, "ssa_testj_fd.sh")))],
    }
    out["test_v_cfbc"] = {
        "script": "test/regression/ssa/ssa_test_cfbc.sh:25-45",
        "options": {"My": 3, "ksp": "richardson + lu (direct)", "mpi_ranks": 1},
        "cases": [dict(Mx=M, My=3, **row) for M, row in zip((201, 401), parse_error_tables(
            os.path.join(ssa, "ssa_test_cfbc.sh")))],
    }
    # the SSAFEM regression tables (ssa_method fem, -ksp_type cg, 2 ranks)
    for key, script, sizes in (("test_i_fem", "ssa_testi_fem.sh", ((5, 61), (5, 121))),
                               ("test_j_fem", "ssa_testj_fem.sh", ((61, 61), (121, 121))),
                               ("linear_fem", "ssafem_test_linear.sh", ((61, 61), (121, 121))),
                               ("plug_fem", "ssafem_test_plug.sh", ((22, 31), (61, 61)))):
        out[key] = {
            "script": "test/regression/ssa/" + script,
            "options": {"ssa_method": "fem", "ksp_type": "cg", "mpi_ranks": 2},
            "cases": [dict(Mx=Mx, My=My, **row) for (Mx, My), row in zip(sizes, parse_error_tables(
                os.path.join(ssa, script)))],
        }
    # verification table of the user manual
    from scipy.io import netcdf_file
    f = netcdf_file(os.path.join(ref, "doc/verif/I_userman_may2012.nc"), "r", mmap=False)
    tbl = {k: [float(x) for x in f.variables[k].data] for k in
           ("dx", "dy", "max_velocity", "relative_velocity", "maximum_u", "maximum_v", "average_u",
            "average_v")}
    tbl["source"] = "doc/verif/I_userman_may2012.nc (" + f._attributes["source"].decode() + ")"
    tbl["options"] = {"Mx": 5, "ssa_rtol": 5e-7, "ksp_rtol": 1e-12, "note": "test/vfnow.py:293-302,349-350"}
    out["test_i_userman"] = tbl
    f.close()
    # flow-law tables
    out["flow_tables"] = {}
    for law, script in (("gpbld", "test_20.sh"), ("pb", "test_21.sh"), ("hooke", "test_24.sh"),
                        ("arr", "test_26.sh")):
        t = parse_flow_table(os.path.join(ref, "test/regression", script))
        t["script"] = "test/regression/" + script
        out["flow_tables"][law] = t
    # exact solutions from the reference's own C file
    subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={ref}"], check=True,
                   stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(os.path.join(REPO, "oracle/_ref/libexactij.so"))

    class TI(ctypes.Structure):
        _fields_ = [("bed", ctypes.c_double), ("tauc", ctypes.c_double), ("u", ctypes.c_double),
                    ("v", ctypes.c_double)]

    class TJ(ctypes.Structure):
        _fields_ = [("H", ctypes.c_double), ("nu", ctypes.c_double), ("u", ctypes.c_double),
                    ("v", ctypes.c_double)]

    lib.exactI.restype = TI
    lib.exactI.argtypes = [ctypes.c_double] * 3
    lib.exactJ.restype = TJ
    lib.exactJ.argtypes = [ctypes.c_double] * 2
    pts_i = [(x, y) for x in (-60e3, -13e3, 0.0, 30e3, 60e3)
             for y in (-120e3, -47.9e3, -40e3, -12.5e3, 0.0, 3.3e3, 39.999e3, 48.2e3, 120e3)]
    out["exact_i"] = {"m": 10.0, "points": [[x, y, *[getattr(lib.exactI(10.0, x, y), k) for k in
                                                      ("bed", "tauc", "u", "v")]] for x, y in pts_i]}
    pts_j = [(x, y) for x in (-300e3, -150e3, -12.3e3, 0.0, 77e3, 295e3)
             for y in (-300e3, -100e3, 0.0, 5e3, 211e3, 300e3)]
    out["exact_j"] = {"points": [[x, y, *[getattr(lib.exactJ(x, y), k) for k in ("H", "nu", "u", "v")]]
                                 for x, y in pts_j]}
    path = os.path.join(HERE, "reference_goldens.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PISM_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set PISM_REFERENCE_ROOT)")
    main(root)
