"""Test configuration: the gpu marker, the package alias and the oracle's native build.

The package directory is named ``pismv0.7.3_b200`` (not an importable identifier),
so it is registered here under the alias ``pism_b200``.
"""
import importlib.util
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(REPO, "pismv0.7.3_b200")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def _load_package():
    if "pism_b200" in sys.modules:
        return sys.modules["pism_b200"]
    spec = importlib.util.spec_from_file_location(
        "pism_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pism_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    lib = os.path.join(REPO, "oracle", "_build", "libksp_cpu.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), os.path.join(REPO, "oracle", "_build",
                                                                                  "libksp_cpu.so")],
                       check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def goldens():
    import json
    with open(os.path.join(REPO, "tests", "golden", "reference_goldens.json")) as fh:
        return json.load(fh)
