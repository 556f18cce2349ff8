"""SSAFEM on the GPU (pism_gpu_ssafem_solve) against the oracle's converged finite-element
solution (oracle/ssafem_oracle.py) and the reference's SSAFEM regression tables
(test/regression/ssa/ssa_testi_fem.sh, ssa_testj_fem.sh, ssafem_test_linear.sh,
ssafem_test_plug.sh)."""
import json
import os

import numpy as np
import pytest

from pism_b200 import verification as V
from pism_b200.config import GridDesc
from oracle import ssafd_oracle as O
from oracle import ssafem_oracle as F

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pism_b200.ssa import SSAFEM, SSAFEMFailure  # noqa: E402

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_goldens.json")))
COLS = ("maxvector", "prcntavvec", "maxu", "maxv", "avu", "avv")
DIGITS = {"maxvector": 4, "prcntavvec": 5, "maxu": 4, "maxv": 4, "avu": 4, "avv": 4}
CASES = {
    "test_i_fem": lambda Mx, My: (V.build_test_i(My=My, Mx=Mx), lambda g, c: V.exact_velocity_i(g)),
    "test_j_fem": lambda Mx, My: (V.build_test_j(Mx, My), lambda g, c: V.exact_velocity_j(g)),
    "linear_fem": lambda Mx, My: (V.build_test_linear(Mx, My), V.exact_velocity_linear),
    "plug_fem": lambda Mx, My: (V.build_test_plug(Mx, My), V.exact_velocity_plug),
}
TIGHT = dict(snes_rtol=1e-11, ksp_rtol=1e-10, ksp_max_it=100000)


def gpu_solve(g, c, f, **options):
    s = SSAFEM(g, c, **options)
    try:
        s.set_inputs(**{k: f[k] for k in ("thickness", "surface", "bed", "mask", "tauc")},
                     enthalpy=f.get("enthalpy"), bc_mask=f.get("bc_mask"), bc_values=f.get("bc_values"))
        s.set_initial_guess(np.zeros((g.Mx, g.My, 2)))
        return s.solve(), s.stats()
    finally:
        s.close()


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("key,idx", [(k, i) for k in CASES for i in (0, 1)])
def test_regression_tables_with_the_reference_settings(key, idx):
    """SNES / KSP at PETSc's defaults (1e-8 / 1e-5): the printed error table of the reference"""
    row = GOLDEN[key]["cases"][idx]
    (g, c, f), exact = CASES[key](row["Mx"], row["My"])
    vel, st = gpu_solve(g, c, f)
    assert st["converged"] > 0
    r = V.report(vel, exact(g, c))
    for col in COLS:
        assert round(r[col], DIGITS[col]) == pytest.approx(row[col], abs=0.6 * 10.0 ** -DIGITS[col]), col


@pytest.mark.parametrize("key,Mx,My", [("test_i_fem", 5, 61), ("test_j_fem", 61, 61), ("linear_fem", 61, 61),
                                       ("plug_fem", 22, 31)])
def test_matches_the_oracle(key, Mx, My):
    (g, c, f), _ = CASES[key](Mx, My)
    vel, st = gpu_solve(g, c, f, **TIGHT)
    ref, _ = F.SSAFEMOracle(*O.from_case(g, c, f)).solve()
    assert st["converged"] > 0
    assert rel_l2(vel, ref) < 1e-8


def test_enthalpy_hardness_at_the_quadrature_points():
    """test I's stream with the GPBLD flow law on random enthalpy columns: the hardness is the
    column average of the enthalpy interpolated to each quadrature point"""
    g0, c, f = V.build_test_i(My=41, Mx=7)
    g = GridDesc(g0.Mx, g0.My, g0.Lx, g0.Ly, periodicity=0, z=np.linspace(0.0, 2500.0, 11))
    c = c.copy(flow_law="gpbld")
    rng = np.random.default_rng(5)
    f = dict(f, enthalpy=rng.uniform(5.0e4, 1.5e5, (g.Mx, g.My, 11)))
    vel, st = gpu_solve(g, c, f, **TIGHT)
    ref, _ = F.SSAFEMOracle(*O.from_case(g, c, f)).solve()
    assert st["converged"] > 0
    assert rel_l2(vel, ref) < 1e-8


def test_failure_to_converge_raises():
    """too few Newton steps: SSAFEMFailure, and the velocity is the one the solve started from"""
    g, c, f = V.build_test_i(My=61)
    s = SSAFEM(g, c, snes_max_it=1)
    try:
        s.set_inputs(**{k: f[k] for k in ("thickness", "surface", "bed", "mask", "tauc")},
                     bc_mask=f["bc_mask"], bc_values=f["bc_values"])
        start = np.full((g.Mx, g.My, 2), 1e-6)
        s.set_initial_guess(start)
        with pytest.raises(SSAFEMFailure):
            s.solve()
        np.testing.assert_array_equal(s.velocity(), start)
    finally:
        s.close()


def test_the_front_end_builds_ssafem():
    """SSARun with ssa_method "fem" constructs the finite-element solver and solves the plug flow"""
    from pism_b200 import pism_ssa as P
    g, c, f = V.build_test_plug(22, 31)

    class Plug(P.SSAExactTestCase):
        def _initGrid(self):
            self.grid = P.Grid(g)

        def _constructModelData(self):
            cfg = P.Config(c)
            cfg.set_string("ssa_method", "fem")
            return P.ModelData(self.grid, cfg)

        def _initPhysics(self):
            self.modeldata.setPhysics(P.EnthalpyConverter(self.config))

        def _initSSACoefficients(self):
            self._allocStdSSACoefficients()
            self._allocateBCs()
            v = self.modeldata.vecs
            v.land_ice_thickness[:] = f["thickness"]
            v.surface_altitude[:] = f["surface"]
            v.bedrock_altitude[:] = f["bed"]
            v.mask[:] = f["mask"]
            v.bc_mask[:] = f["bc_mask"]
            v.vel_bc[:] = f["bc_values"]

        def exactSolution(self, i, j, x, y):
            return V.exact_velocity_plug(g, c)[i, j]

    case = Plug(g.Mx, g.My)
    r = case.run()
    assert type(case.ssa).__name__ == "SSAFEM"
    row = GOLDEN["plug_fem"]["cases"][0]
    assert round(r["maxu"], 4) == pytest.approx(row["maxu"], abs=6e-5)
    case.ssa.close()
