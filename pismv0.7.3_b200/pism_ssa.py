"""The SSA driver classes of PISM's Python front end over the B200 solver.

PISM's `site-packages/PISM/ssa.py:29-340` lets a script solve the SSA without an IceModel:
`SSARun.setup()` runs the hooks `_setFromOptions`, `_initGrid`, `_constructModelData`,
`_initPhysics`, `_constructSSA`, `_initSSACoefficients`, `_initSSA` in that order,
`solve()` calls the SSA's `update`, and `SSAExactTestCase` adds `run`, `report` (the
verification table of SSATestCase::report) and `exactSolution`.  This module keeps those
names, the order of the hooks and the names of the model vectors
(`land_ice_thickness`, `bedrock_altitude`, `surface_altitude`, `tauc`, `enthalpy`, `mask`,
`bc_mask`, `vel_bc`; `site-packages/PISM/model.py`), so a test case written for the
reference's front end reads the same against this one.  The vectors are numpy arrays
indexed [i, j] (velocities [i, j, 2]); `Grid.Shallow` stands for `PISM.IceGrid.Shallow`, the
configuration for PISM's `Config` (the names of `pism_config.cdl`, stored in the solver's
`SSAConfig`), and `write` stores the vectors and the solution in an `.npz` file where the
reference writes NetCDF.
"""
from __future__ import annotations

import numpy as np

from .config import SSAConfig, GridDesc
from .verification import report as _report, SECPERA

# pism_config.cdl names whose solver field is spelt differently
_ALIASES = {"ssa_flow_law": "flow_law", "Glen_exponent": "ssa_Glen_exponent"}

MASK_ICE_FREE_BEDROCK, MASK_GROUNDED, MASK_FLOATING, MASK_ICE_FREE_OCEAN = 0, 2, 3, 4   # Mask.hh:28-34


class Config:
    """PISM's Config (get_* / set_* by pism_config.cdl name) over the solver's SSAConfig."""

    def __init__(self, cfg: SSAConfig | None = None):
        self.cfg = (cfg or SSAConfig()).copy()
        self.ssa_method = "fd"

    def _field(self, name):
        f = _ALIASES.get(name, name)
        if not hasattr(self.cfg, f):
            raise KeyError(f"unknown configuration parameter {name}")
        return f

    def get_double(self, name):
        return float(getattr(self.cfg, self._field(name)))

    def get_boolean(self, name):
        return bool(getattr(self.cfg, self._field(name)))

    def get_string(self, name):
        if name == "ssa_method":
            return self.ssa_method
        return str(getattr(self.cfg, self._field(name)))

    def set_double(self, name, value):
        setattr(self.cfg, self._field(name), float(value))

    def set_boolean(self, name, value):
        setattr(self.cfg, self._field(name), bool(value))

    def set_string(self, name, value):
        if name == "ssa_method":
            if value not in ("fd", "fem", "gpu"):
                raise ValueError(f"unknown ssa_method {value} (fd or fem)")
            self.ssa_method = value
            return
        setattr(self.cfg, self._field(name), value)


class Grid:
    """PISM.IceGrid's horizontal geometry (IceGrid.cc:540-610) for the SSA: Mx, My, x(i),
    y(j), dx, dy and points()."""

    def __init__(self, desc: GridDesc):
        self.desc = desc
        self._x, self._y = desc.x_coords(), desc.y_coords()

    @classmethod
    def Shallow(cls, Lx, Ly, x0, y0, Mx, My, periodicity=0):
        """IceGrid::Shallow (IceGrid.cc:148-176): half-widths Lx, Ly around (x0, y0)."""
        return cls(GridDesc.shallow(Mx, My, Lx, Ly, periodicity=periodicity, x0=x0, y0=y0))

    def Mx(self):
        return self.desc.Mx

    def My(self):
        return self.desc.My

    def x(self, i):
        return float(self._x[i])

    def y(self, j):
        return float(self._y[j])

    def dx(self):
        return self.desc.dx

    def dy(self):
        return self.desc.dy

    def points(self):
        for i in range(self.desc.Mx):
            for j in range(self.desc.My):
                yield i, j


class Vecs:
    """PISM.model.ModelVecs: named model vectors, reachable as attributes."""

    def __init__(self):
        self._names = []

    def add(self, array, name):
        setattr(self, name, array)
        self._names.append(name)

    def has(self, name):
        return name in self._names

    def names(self):
        return list(self._names)


class ModelData:
    """PISM.model.ModelData: grid, configuration, vectors and the physics objects."""

    def __init__(self, grid: Grid, config: Config | None = None):
        self.grid = grid
        self.config = config or Config()
        self.vecs = Vecs()
        self.enthalpyconverter = None

    def setPhysics(self, enthalpyconverter):
        self.enthalpyconverter = enthalpyconverter


class EnthalpyConverter:
    """Stands for PISM.EnthalpyConverter: its constants are the configuration's."""

    def __init__(self, config: Config):
        self.config = config


class SSARun:
    """site-packages/PISM/ssa.py:29-225 over the B200 SSAFD."""

    def __init__(self):
        self.grid = None
        self.config = None
        self.modeldata = None
        self.ssa = None

    def setup(self):
        self._setFromOptions()
        self._initGrid()
        if self.grid is None:
            raise RuntimeError("SSARun failed to provide a grid.")
        self.modeldata = self._constructModelData()
        if self.modeldata is None:
            raise RuntimeError("SSARun._constructModelData failed to provide a ModelData.")
        self.config = self.modeldata.config
        self._initPhysics()
        if self.modeldata.enthalpyconverter is None:
            raise RuntimeError("SSARun._initPhysics failed to initialize the physics of the underlying SSA solver.")
        self.ssa = self._constructSSA()
        if self.ssa is None:
            raise RuntimeError("SSARun._constructSSA failed to provide an SSA.")
        self._initSSACoefficients()
        self._initSSA()

    def solve(self):
        """SSA::update with fast = false on the model vectors; returns the velocity [Mx, My, 2]."""
        v = self.modeldata.vecs
        shape = (self.grid.Mx(), self.grid.My())
        fields = {"thickness": v.land_ice_thickness, "surface": v.surface_altitude, "bed": v.bedrock_altitude,
                  "mask": v.mask, "tauc": v.tauc,
                  "melange": v.melange_back_pressure if v.has("melange_back_pressure") else np.zeros(shape)}
        if v.has("enthalpy") and self.config.get_string("ssa_flow_law") != "isothermal_glen":
            fields["enthalpy"] = v.enthalpy
        bc = {}
        if v.has("vel_bc") and v.has("bc_mask"):
            bc = {"bc_mask": v.bc_mask, "bc_values": v.vel_bc}
        # the configuration as the script left it; the strength extension is the solver's own
        # member (SSA::strength_extension), as in PISM
        se = self.ssa.config.min_thickness_strength_extension_ssa
        self.ssa.set_config(self.config.cfg.copy(min_thickness_strength_extension_ssa=se))
        self.ssa.set_inputs(**fields, **bc)
        self.ssa.update(False)
        self.velocity = self.ssa.velocity()
        return self.velocity

    def write(self, filename):
        """The model vectors and the solution ("velbar") in an .npz file."""
        v = self.modeldata.vecs
        np.savez(filename, velbar=self.ssa.velocity(), **{n: getattr(v, n) for n in v.names()})

    # hooks
    def _setFromOptions(self):
        pass

    def _constructModelData(self):
        return ModelData(self.grid)

    def _initGrid(self):
        raise NotImplementedError()

    def _initPhysics(self):
        raise NotImplementedError()

    def _allocStdSSACoefficients(self):
        """surface, thickness, bed, tauc, enthalpy and mask (ssa.py:165-190)."""
        v = self.modeldata.vecs
        shape = (self.grid.Mx(), self.grid.My())
        Mz = 0 if self.grid.desc.z is None else len(self.grid.desc.z)
        v.add(np.zeros(shape), "surface_altitude")
        v.add(np.zeros(shape), "land_ice_thickness")
        v.add(np.zeros(shape), "bedrock_altitude")
        v.add(np.zeros(shape), "tauc")
        v.add(np.zeros((*shape, max(Mz, 1))), "enthalpy")
        v.add(np.zeros(shape), "mask")

    def _allocateBCs(self, velname="_bc", maskname="bc_mask"):
        """vel_bc and bc_mask (ssa.py:192-208)."""
        v = self.modeldata.vecs
        shape = (self.grid.Mx(), self.grid.My())
        v.add(np.zeros((*shape, 2)), "vel_bc")
        v.add(np.zeros(shape), "bc_mask")

    def _initSSACoefficients(self):
        raise NotImplementedError()

    def _constructSSA(self):
        """SSAFD on the B200, or SSAFEM with ssa_method "fem" (PISM/ssa.py's SSAFactory choice)."""
        from .ssa import SSAFD, SSAFEM
        if self.config.get_string("ssa_method") == "fem":
            return SSAFEM(self.grid.desc, self.config.cfg)
        return SSAFD(self.grid.desc, self.config.cfg)

    def _initSSA(self):
        pass


class SSAExactTestCase(SSARun):
    """site-packages/PISM/ssa.py:226-338: a test case with an exact solution."""

    def __init__(self, Mx, My):
        SSARun.__init__(self)
        self.Mx = Mx
        self.My = My

    def run(self, output_file=None):
        self.setup()
        self.solve()
        table = self.report()
        if output_file:
            self.write(output_file)
        return table

    def exact_velocity(self):
        """exactSolution at every cell, [Mx, My, 2] (m/s)."""
        out = np.zeros((self.grid.Mx(), self.grid.My(), 2))
        for i, j in self.grid.points():
            out[i, j] = self.exactSolution(i, j, self.grid.x(i), self.grid.y(j))
        return out

    def report(self):
        """SSATestCase::report: the error table in m/year and percent, printed as the
        reference prints it; returns it as a dict."""
        r = _report(self.ssa.velocity(), self.exact_velocity())
        print("NUMERICAL ERRORS in velocity relative to exact solution:")
        print("velocity  :  maxvector   prcntavvec      maxu      maxv       avu       avv")
        print("           %11.4f%13.5f%10.4f%10.4f%10.4f%10.4f" % (
            r["maxvector"], r["prcntavvec"], r["maxu"], r["maxv"], r["avu"], r["avv"]))
        print("NUM ERRORS DONE")
        return r

    def exactSolution(self, i, j, x, y):
        raise NotImplementedError()

    def write(self, filename):
        v = self.modeldata.vecs
        np.savez(filename, velbar=self.ssa.velocity(), vel_exact=self.exact_velocity(),
                 **{n: getattr(v, n) for n in v.names()})


__all__ = ["Config", "Grid", "Vecs", "ModelData", "EnthalpyConverter", "SSARun", "SSAExactTestCase", "SECPERA",
           "MASK_ICE_FREE_BEDROCK", "MASK_GROUNDED", "MASK_FLOATING", "MASK_ICE_FREE_OCEAN"]
