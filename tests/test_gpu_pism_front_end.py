"""The Python front end's SSAExactTestCase (site-packages/PISM/ssa.py:226-338) driving the B200
solver: Schoof's plug flow down a uniform slope with no basal resistance and Dirichlet edges
(an exact solution; the reference's examples/python/ssa_tests/ssa_test_plug.py sets up the same
physics), against the oracle on the same inputs and against the exact solution at two
resolutions (second-order convergence)."""
import numpy as np
import pytest

from pism_b200 import pism_ssa as P
from pism_b200.verification import report
from oracle import ssafd_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)


class Plug(P.SSAExactTestCase):
    """plug flow: thickness H0, surface and bed sloping at dhdx in x, no basal resistance,
    hardness B0, exact speed u(y) = f^3 L^4 (1 - (y / L)^4) / (2 (B0 H0)^3), f = rho g H0 dhdx"""
    H0, L, dhdx, B0, n = 2000.0, 50e3, 0.001, 3.7e8, 3.0

    def _initGrid(self):
        self.grid = P.Grid.Shallow(self.L, self.L, 0, 0, self.Mx, self.My)

    def _initPhysics(self):
        self.config.set_string("ssa_flow_law", "isothermal_glen")
        self.config.set_double("ice_softness", self.B0 ** -self.n)
        self.config.set_double("Glen_exponent", self.n)
        self.modeldata.setPhysics(P.EnthalpyConverter(self.config))

    def _initSSACoefficients(self):
        self._allocStdSSACoefficients()
        self._allocateBCs()
        v, g = self.modeldata.vecs, self.grid
        v.land_ice_thickness[:] = self.H0
        v.tauc[:] = 0.0
        v.mask[:] = P.MASK_GROUNDED
        for i, j in g.points():
            x, y = g.x(i), g.y(j)
            v.bedrock_altitude[i, j] = -x * self.dhdx
            v.surface_altitude[i, j] = v.bedrock_altitude[i, j] + self.H0
            if i in (0, g.Mx() - 1) or j in (0, g.My() - 1):
                v.bc_mask[i, j] = 1
                v.vel_bc[i, j] = self.exactSolution(i, j, x, y)

    def _initSSA(self):
        self.ssa.strength_extension.set_min_thickness(self.H0 / 2)
        self.config.set_double("epsilon_ssa", 0.0)
        self.config.set_double("ssafd_relative_convergence", 1e-7)
        self.config.set_double("ksp_rtol", 1e-12)

    def exactSolution(self, i, j, x, y):
        f = self.config.get_double("ice_density") * self.config.get_double("standard_gravity") * self.H0 * self.dhdx
        return [0.5 * f ** 3 * self.L ** 4 / (self.B0 * self.H0) ** 3 * (1.0 - (y / self.L) ** 4), 0.0]


def oracle_velocity(case):
    v = case.modeldata.vecs
    M = (case.grid.Mx(), case.grid.My())
    f = {"thickness": v.land_ice_thickness, "surface": v.surface_altitude, "bed": v.bedrock_altitude,
         "mask": v.mask, "tauc": v.tauc, "bc_mask": v.bc_mask, "bc_values": v.vel_bc, "melange": np.zeros(M)}
    cfg = case.config.cfg.copy(min_thickness_strength_extension_ssa=case.H0 / 2)
    return O.SSAFDOracle(*O.from_case(case.grid.desc, cfg, f)).solve()


def test_plug_flow_through_the_front_end(capsys):
    errs = {}
    for M in (31, 61):
        case = Plug(M, M)
        table = case.run()
        ref = oracle_velocity(case)
        vel = case.ssa.velocity()
        assert np.linalg.norm(vel - ref) / np.linalg.norm(ref) < 1e-8
        ref_table = report(ref, case.exact_velocity())
        # the table prints m/year to 4 decimals (SSATestCase::report); the two velocities agree
        # to 1e-8 of a 1400 m/year flow, so the printed errors agree to those digits
        for k in ("maxvector", "maxu", "avu"):
            assert table[k] == pytest.approx(ref_table[k], abs=1e-4), k
        errs[M] = table["maxvector"]
        case.ssa.close()
    assert 3.5 < errs[31] / errs[61] < 4.5   # second order
    assert "NUM ERRORS DONE" in capsys.readouterr().out
