"""The Python front end's SSA driver classes (pism_b200.pism_ssa: SSARun, SSAExactTestCase,
site-packages/PISM/ssa.py:29-338) on CPU: the order of the set-up hooks, the configuration by
pism_config.cdl names, the model vectors and the error table, with a stand-in solver."""
import numpy as np
import pytest

from pism_b200 import pism_ssa as P


class FakeSSA:
    """records what the front end hands the solver"""

    def __init__(self, grid, config):
        self.config = config.copy()
        self.calls = []
        self.vel = None

    def set_config(self, c):
        self.config = c.copy()
        self.calls.append("set_config")

    def set_inputs(self, **kw):
        self.inputs = kw
        self.calls.append("set_inputs")

    def update(self, fast):
        self.calls.append(("update", fast))
        self.vel = np.zeros((*self.inputs["thickness"].shape, 2))
        self.vel[..., 0] = 1.0 / P.SECPERA   # 1 m/year everywhere

    def velocity(self):
        return self.vel


class Case(P.SSAExactTestCase):
    order = []

    def _setFromOptions(self):
        self.order.append("options")

    def _initGrid(self):
        self.order.append("grid")
        self.grid = P.Grid.Shallow(50e3, 40e3, 0, 0, self.Mx, self.My)

    def _initPhysics(self):
        self.order.append("physics")
        self.config.set_string("ssa_flow_law", "isothermal_glen")
        self.config.set_double("ice_softness", 3.7e8 ** -3)
        self.config.set_double("Glen_exponent", 3.0)
        self.modeldata.setPhysics(P.EnthalpyConverter(self.config))

    def _constructSSA(self):
        self.order.append("ssa")
        return FakeSSA(self.grid.desc, self.config.cfg)

    def _initSSACoefficients(self):
        self.order.append("coefficients")
        self._allocStdSSACoefficients()
        self._allocateBCs()
        v = self.modeldata.vecs
        v.land_ice_thickness[:] = 1000.0
        v.mask[:] = P.MASK_GROUNDED
        v.bc_mask[0, :] = 1

    def _initSSA(self):
        self.order.append("init")
        self.config.set_double("epsilon_ssa", 0.0)

    def exactSolution(self, i, j, x, y):
        return [1.0 / P.SECPERA * (1.0 + (i == 0)), 0.0]


def test_hooks_run_in_the_reference_order_and_feed_the_solver(tmp_path, capsys):
    c = Case(7, 5)
    table = c.run(str(tmp_path / "out.npz"))
    assert Case.order == ["options", "grid", "physics", "ssa", "coefficients", "init"]
    s = c.ssa
    assert s.calls[-1] == ("update", False)
    assert s.config.flow_law == "isothermal_glen" and s.config.ssa_Glen_exponent == 3.0 and s.config.epsilon_ssa == 0.0
    assert s.inputs["thickness"].shape == (7, 5) and "bc_mask" in s.inputs and "enthalpy" not in s.inputs
    # one column is off by 1 m/year: max 1, average 5/35 m/year, 5/35 of the largest exact speed 2 m/year
    assert table["maxu"] == pytest.approx(1.0) and table["avu"] == pytest.approx(5 / 35)
    assert table["prcntavvec"] == pytest.approx(5 / 35 / 2.0 * 100.0)
    out = capsys.readouterr().out
    assert "maxvector   prcntavvec      maxu      maxv       avu       avv" in out
    saved = np.load(tmp_path / "out.npz")
    assert {"velbar", "vel_exact", "land_ice_thickness", "bc_mask"} <= set(saved.files)


def test_config_names_and_grid():
    cfg = P.Config()
    cfg.set_double("ssafd_relative_convergence", 1e-5)
    assert cfg.get_double("ssafd_relative_convergence") == 1e-5
    cfg.set_boolean("ssa_dirichlet_bc", True)
    assert cfg.get_boolean("ssa_dirichlet_bc")
    assert cfg.get_string("ssa_method") == "fd"
    cfg.set_string("ssa_method", "fem")   # SSAFEM, the finite-element solver
    assert cfg.get_string("ssa_method") == "fem"
    with pytest.raises(ValueError):
        cfg.set_string("ssa_method", "spectral")
    with pytest.raises(KeyError):
        cfg.get_double("no_such_parameter")
    g = P.Grid.Shallow(10e3, 5e3, 0, 0, 11, 6)
    assert g.x(0) == -10e3 and g.x(10) == 10e3 and g.dx() == 2e3 and g.y(5) == 5e3
    assert len(list(g.points())) == 66
