"""The C++ host path (SSAFD_GPU + ssa_test_gpu) against the reference's regression scripts.

ssa_test_gpu prints SSATestCase::report's table; its lines must equal the expected
output recorded in test/regression/ssa/ssa_testi_fd.sh and ssa_test_cfbc.sh."""
import os
import subprocess

import numpy as np

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(REPO, "pismv0.7.3_b200", "lib", "ssa_test_gpu")


def table_line(row):
    return "           %11.4f%13.5f%10.4f%10.4f%10.4f%10.4f" % (
        row["maxvector"], row["prcntavvec"], row["maxu"], row["maxv"], row["avu"], row["avv"])


def run(*args):
    r = subprocess.run([EXE, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0] == "NUMERICAL ERRORS in velocity relative to exact solution:"
    assert lines[3] == "NUM ERRORS DONE"
    return lines[2]


@pytest.mark.parametrize("pc", ["mg", "bjacobi", "line"])
@pytest.mark.parametrize("k", [0, 1])
def test_driver_test_i(goldens, k, pc):
    case = goldens["test_i_fd"]["cases"][k]
    got = run("-test", "I", "-My", str(case["My"]), "-ssa_rtol", "5e-07", "-ssafd_ksp_rtol", "1e-12", "-pc", pc)
    assert got == table_line(case)


@pytest.mark.parametrize("k", [0, 1])
def test_driver_test_v(goldens, k):
    case = goldens["test_v_cfbc"]["cases"][k]
    got = run("-test", "V", "-Mx", str(case["Mx"]), "-My", "3", "-ssafd_ksp_rtol", "1e-13")
    assert got == table_line(case)


def test_driver_learned_warm_start(tmp_path):
    """SSAFD_GPU::set_warm_start: starting test I from the learned guess ends at the same
    answer once the Picard tolerance is tight: the tables agree to within one unit of their
    last printed digit (two answers 1e-9 apart may round either side of a printed digit)."""
    import re
    params = np.load(os.path.join(REPO, "pismv0.7.3_b200", "weights", "unet_ssa_10km.npz"))["params"]
    f32 = tmp_path / "unet.f32"
    params.astype(np.float32).tofile(f32)
    args = ("-test", "I", "-My", "61", "-ssa_rtol", "1e-9", "-ssafd_ksp_rtol", "1e-12")
    a, b = run(*args, "-learned", str(f32)), run(*args)
    na, nb = re.findall(r"-?\d+\.\d+", a), re.findall(r"-?\d+\.\d+", b)
    assert len(na) == len(nb) > 0
    for x, y in zip(na, nb):
        unit = 10.0 ** -len(x.split(".")[1])
        assert abs(float(x) - float(y)) <= 1.01 * unit, (x, y)
