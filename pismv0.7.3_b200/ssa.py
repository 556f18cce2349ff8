"""Host-side mirror of PISM's SSA interface over the B200 C-ABI.

``SSAFD`` keeps the names, argument meaning and error behaviour of the
reference's ``pism::stressbalance::SSAFD`` (src/base/stressbalance/ssa/SSAFD.hh,
SSA.hh:110-156, ShallowStressBalance.hh:39-99): ``init``, ``update(fast,
melange_back_pressure)``, ``solve``, ``set_boundary_conditions``,
``set_initial_guess``, ``velocity``, ``basal_frictional_heating``,
``stdout_report``, and the stage methods ``assemble_rhs``,
``compute_hardav_staggered``, ``compute_nuH_staggered``.  Failures raise
``RuntimeError`` subclasses named as in the reference (``KSPFailure``,
``PicardFailure``, SSAFD.hh:115-123).

Arrays are numpy FP64 arrays indexed ``[i, j]`` (``[..., 2]`` for vectors) or,
to keep data on the device, CUDA tensors of the same shape (``torch.float64``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from .config import CFemOptions, CFemStats, CInputs, CMember, CStats, GridDesc, SSAConfig

_D = C.POINTER(C.c_double)


class SSAError(RuntimeError):
    """RuntimeError raised by the solver (pism::RuntimeError)."""


class KSPFailure(SSAError):
    """SSAFD::KSPFailure (SSAFD.hh:115-118)."""


class PicardFailure(SSAError):
    """SSAFD::PicardFailure (SSAFD.hh:120-123)."""


class ZeroDiagonal(SSAError):
    """Zero diagonal entry at a regular location (SSAFD.cc:766-776)."""


_EXC = {_capi.EKSP: KSPFailure, _capi.EPICARD: PicardFailure, _capi.EZERODIAG: ZeroDiagonal}


def _is_device(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


class _Buf:
    """Pointer + keep-alive for a host numpy array or a CUDA tensor."""

    def __init__(self, a, shape):
        if a is None:
            self.ptr, self.keep, self.device = None, None, None
            return
        if _is_device(a):
            import torch
            t = a.to(torch.float64).contiguous()
            if tuple(t.shape) != tuple(shape):
                t = t.reshape(shape)
            if t.data_ptr() != a.data_ptr():
                # the converted copy was written on torch's current stream; the library reads
                # it on the handle's stream, which does not wait for that one
                torch.cuda.current_stream(t.device).synchronize()
            self.keep, self.device = t, True
            self.ptr = C.cast(C.c_void_p(t.data_ptr()), _D)
        else:
            arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))
            self.keep, self.device = arr, False
            self.ptr = arr.ctypes.data_as(_D)


class SSAFD:
    """B200 finite-difference SSA solver with the reference's SSAFD interface."""

    def __init__(self, grid: GridDesc, config: SSAConfig | None = None, device: int = 0):
        self.lib = _capi.load()
        self.grid = grid
        self.config = (config or SSAConfig()).copy()
        self.device = device
        self._h = C.c_void_p()
        cgrid, self._z = grid.to_c()
        ccfg = self.config.to_c()
        rc = self.lib.pism_gpu_ssa_create(C.byref(cgrid), C.byref(ccfg), device, C.byref(self._h))
        if rc != _capi.OK:
            raise SSAError(f"pism_gpu_ssa_create failed with status {rc}")
        self._stats = CStats()
        self._bc = (None, None)
        self._fields = {}
        self._stdout = ""

    # ---- lifetime ----
    def close(self):
        if self._h:
            self.lib.pism_gpu_ssa_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != _capi.OK:
            msg = self.lib.pism_gpu_ssa_last_error(self._h).decode() or what
            raise _EXC.get(rc, SSAError)(f"{what}: {msg} (status {rc})")

    @property
    def shape(self):
        return (self.grid.Mx, self.grid.My)

    # ---- configuration and inputs ----
    def set_config(self, config: SSAConfig):
        self.config = config.copy()
        ccfg = self.config.to_c()
        self._check(self.lib.pism_gpu_ssa_set_config(self._h, C.byref(ccfg)), "set_config")

    def set_stream(self, cuda_stream_ptr: int | None):
        self._check(self.lib.pism_gpu_ssa_set_stream(self._h, C.c_void_p(cuda_stream_ptr or 0)), "set_stream")

    def init(self):
        """SSAFD::init_impl: nothing to fetch; inputs come through set_inputs."""

    def set_boundary_conditions(self, locations, velocities):
        """ShallowStressBalance::set_boundary_conditions(bc_mask, vel_ssa_bc)."""
        self._bc = (locations, velocities)
        if self._fields:
            self._upload()

    def set_inputs(self, thickness, surface, bed, mask, tauc, melange=None, gl_mask=None, enthalpy=None,
                   hardness=None, fracture_density=None, bc_mask=None, bc_values=None):
        """Hand over the fields SSA::init_impl fetches by name (SSA.cc:134-184)."""
        self._fields = dict(thickness=thickness, surface=surface, bed=bed, mask=mask, tauc=tauc,
                            melange=melange, gl_mask=gl_mask, enthalpy=enthalpy, hardness=hardness,
                            fracture_density=fracture_density)
        if bc_mask is not None:
            self._bc = (bc_mask, bc_values)
        self._upload()

    def _inputs(self, f, bc):
        """the C inputs struct of the fields f (and bc = (bc_mask, bc_values)) plus the
        buffers that keep them alive"""
        Mx, My = self.shape
        Mz = 0 if self.grid.z is None else len(self.grid.z)
        s2, s3 = (Mx, My), (Mx, My, 2)
        bufs = {
            "thickness": _Buf(f["thickness"], s2), "surface": _Buf(f["surface"], s2),
            "bed": _Buf(f["bed"], s2), "mask": _Buf(f["mask"], s2), "tauc": _Buf(f["tauc"], s2),
            "bc_mask": _Buf(bc[0], s2), "bc_values": _Buf(bc[1], s3),
            "melange": _Buf(f.get("melange"), s2), "gl_mask": _Buf(f.get("gl_mask"), s2),
            "enthalpy": _Buf(f.get("enthalpy"), (Mx, My, Mz)), "hardness_stag": _Buf(f.get("hardness"), s3),
            "fracture_density": _Buf(f.get("fracture_density"), s2),
        }
        kinds = {b.device for b in bufs.values() if b.ptr is not None}
        if len(kinds) > 1:
            raise ValueError("inputs must be all host arrays or all CUDA tensors")
        ci = CInputs()
        ci.where = _capi.MEM_DEVICE if kinds == {True} else _capi.MEM_HOST
        for name, b in bufs.items():
            setattr(ci, name, b.ptr)
        return ci, bufs

    def _upload(self):
        ci, _keep = self._inputs(self._fields, self._bc)
        self._check(self.lib.pism_gpu_ssa_set_inputs(self._h, C.byref(ci)), "set_inputs")

    def solve_batch(self, members, net=None, stride: int = 1):
        """pism_gpu_ssa_solve_batch: members is a list of dicts with the set_inputs fields
        and optionally "ice_softness" and "velocity" (initial guess; output array or CUDA
        tensor).  Returns (velocities, stats) per member; a member whose solve failed has
        stats["status"] != 0."""
        n = len(members)
        arr = (CMember * max(n, 1))()
        stats = (CStats * max(n, 1))()
        keep, outs = [], []
        for q, m in enumerate(members):
            f = {k: m.get(k) for k in ("thickness", "surface", "bed", "mask", "tauc", "melange", "gl_mask",
                                       "enthalpy", "hardness", "fracture_density")}
            ci, bufs = self._inputs(f, (m.get("bc_mask"), m.get("bc_values")))
            device = ci.where == _capi.MEM_DEVICE
            vel = m.get("velocity")
            if vel is None:
                if device:
                    import torch
                    vel = torch.zeros((*self.shape, 2), dtype=torch.float64, device=f["thickness"].device)
                else:
                    vel = np.zeros((*self.shape, 2))
            vb = _Buf(vel, (*self.shape, 2))
            if vb.device != device:
                raise ValueError("a member's velocity must live where its inputs live")
            arr[q].inputs = ci
            arr[q].ice_softness = float(m.get("ice_softness", 0.0))
            arr[q].velocity = vb.ptr
            keep += [bufs, vb]
            outs.append(vb.keep)
        nh = net._h if net is not None else None
        rc = self.lib.pism_gpu_ssa_solve_batch(self._h, nh, stride, n, arr, stats)
        if rc not in (_capi.OK, _capi.EKSP, _capi.EPICARD, _capi.ENAN, _capi.EZERODIAG):
            self._check(rc, "solve_batch")
        return outs, [stats[q].as_dict() for q in range(n)]

    def set_initial_guess(self, guess):
        """SSA::set_initial_guess (SSA.cc:361-363)."""
        b = _Buf(guess, (*self.shape, 2))
        where = _capi.MEM_DEVICE if b.device else _capi.MEM_HOST
        self._check(self.lib.pism_gpu_ssa_set_initial_guess(self._h, b.ptr, where), "set_initial_guess")

    # ---- the solve ----
    def update(self, fast: bool = False, melange_back_pressure=None):
        """SSA::update (SSA.cc:188-196) / SSAFD::update (SSAFD.cc:260-264)."""
        if melange_back_pressure is not None:
            self._fields["melange"] = melange_back_pressure
            self._upload()
        if not fast:
            self.solve()

    def solve(self, out=None):
        """SSAFD::solve (SSAFD.cc:869-924). Returns the velocity ([Mx, My, 2])."""
        if out is None:
            out = np.empty((*self.shape, 2))
        b = _Buf(out, (*self.shape, 2))
        where = _capi.MEM_DEVICE if b.device else _capi.MEM_HOST
        rc = self.lib.pism_gpu_ssa_solve(self._h, b.ptr, where, C.byref(self._stats))
        self._check(rc, "SSAFD solve")
        s = self._stats
        self._stdout = "%5d outer iterations, ~%3.1f KSP iterations each\n" % (
            s.picard_iterations, s.ksp_iterations / max(1, s.picard_iterations))
        return b.keep if b.device else out

    def stats(self) -> dict:
        return self._stats.as_dict()

    def stdout_report(self) -> str:
        return self._stdout

    # ---- fields ----
    def _get(self, field, shape, out=None):
        if out is None:
            out = np.empty(shape)
        b = _Buf(out, shape)
        where = _capi.MEM_DEVICE if b.device else _capi.MEM_HOST
        self._check(self.lib.pism_gpu_ssa_get_field(self._h, field, b.ptr, where), "get_field")
        return b.keep if b.device else out

    def velocity(self, out=None):
        return self._get(_capi.FIELD_VELOCITY, (*self.shape, 2), out)

    def driving_stress(self, out=None):
        return self._get(_capi.FIELD_TAUD, (*self.shape, 2), out)

    def rhs(self, out=None):
        return self._get(_capi.FIELD_RHS, (*self.shape, 2), out)

    def hardness(self, out=None):
        return self._get(_capi.FIELD_HARDNESS, (*self.shape, 2), out)

    def nuH(self, out=None):
        return self._get(_capi.FIELD_NUH, (*self.shape, 2), out)

    def beta(self, out=None):
        return self._get(_capi.FIELD_BETA, self.shape, out)

    def basal_frictional_heating(self, out=None):
        return self._get(_capi.FIELD_BFRICT, self.shape, out)

    def stress_balance_3d(self, basal_melt_rate=None, out=None, device: bool = False) -> dict:
        """The consumers of the velocity in StressBalance::update with a full update
        (PISMStressBalance.cc:79-116): ConstantInColumn's 3-D horizontal velocity "u", "v"
        (SSB_Modifier.cc:126-152), the vertical velocity "w" (PISMStressBalance.cc:192-287; w at
        the base = -basal_melt_rate, or 0 without one) and the volumetric strain heating
        "strain_heating" (PISMStressBalance.cc:369-499), each [Mx, My, Mz], from the current
        velocity.  `out` may give preallocated host arrays or CUDA tensors (all of one kind)
        for any of the four; the others are created (CUDA tensors when device=True)."""
        Mz = 0 if self.grid.z is None else len(self.grid.z)
        shape = (*self.shape, Mz)
        names = ("u", "v", "w", "strain_heating")
        out = dict(out or {})
        on_device = device or any(_is_device(a) for a in out.values())
        for k in names:
            if k not in out:
                if on_device:
                    import torch
                    out[k] = torch.empty(shape, dtype=torch.float64, device=f"cuda:{self.device}")
                else:
                    out[k] = np.empty(shape)
        bufs = {k: _Buf(out[k], shape) for k in names}
        bmr = _Buf(basal_melt_rate, self.shape) if basal_melt_rate is not None else None
        if bmr is not None and bmr.device != on_device:
            raise ValueError("basal_melt_rate must be where the outputs are (host or device)")
        where = _capi.MEM_DEVICE if on_device else _capi.MEM_HOST
        self._check(self.lib.pism_gpu_ssa_stress_balance_3d(
            self._h, bmr.ptr if bmr is not None else None, *(bufs[k].ptr for k in names), where),
            "stress_balance_3d")
        return {k: (bufs[k].keep if on_device else out[k]) for k in names}

    MASS_TOTALS = ("grounded_basal_ice_flux", "nonneg_rule_flux", "sub_shelf_ice_flux", "surface_ice_flux",
                   "sum_divQ_SIA", "sum_divQ_SSA", "Href_to_H_flux", "H_to_Href_flux")

    def mass_continuity_step(self, dt: float, climatic_mass_balance, basal_melt_rate=None, cell_area=None,
                             device: bool = False) -> dict:
        """IceModel::massContExplicitStep (iMgeometry.cc:497-819) over dt seconds from the
        current velocity (ConstantInColumn: no diffusive flux; part_grid off), then
        updateSurfaceElevationAndMask: returns the new "thickness", "mask", "surface", the
        "flux_divergence" and the step's flux "totals" (kg).  Inputs host arrays or CUDA
        tensors (all of one kind); outputs of the same kind."""
        on_device = device or _is_device(climatic_mass_balance)
        shape = self.shape
        if on_device:
            import torch
            out = {k: torch.empty(shape, dtype=torch.float64, device=f"cuda:{self.device}")
                   for k in ("thickness", "mask", "surface", "flux_divergence")}
        else:
            out = {k: np.empty(shape) for k in ("thickness", "mask", "surface", "flux_divergence")}
        ins = [_Buf(a, shape) if a is not None else None for a in (climatic_mass_balance, basal_melt_rate, cell_area)]
        if any(b is not None and b.device != on_device for b in ins):
            raise ValueError("the inputs must all be host arrays or all CUDA tensors")
        outs = {k: _Buf(v, shape) for k, v in out.items()}
        totals = (C.c_double * 8)()
        where = _capi.MEM_DEVICE if on_device else _capi.MEM_HOST
        self._check(self.lib.pism_gpu_ssa_mass_continuity_step(
            self._h, float(dt), *(b.ptr if b is not None else None for b in ins),
            float(self.config.mask_icefree_thickness_standard), float(self.config.mask_is_floating_thickness_standard),
            outs["thickness"].ptr, outs["mask"].ptr, outs["surface"].ptr, outs["flux_divergence"].ptr,
            C.cast(totals, _D), where), "massContExplicitStep")
        res = {k: (outs[k].keep if on_device else out[k]) for k in out}
        res["totals"] = dict(zip(self.MASS_TOTALS, list(totals)))
        return res

    def strain_rates(self, mask=None, edot: bool = True, stresses: bool = True, device: bool = False) -> dict:
        """ShallowStressBalance::compute_2D_principal_strain_rates and compute_2D_stresses
        (ShallowStressBalance.cc:224-386) of the current velocity on `mask` (None: the
        inputs' mask): "edot" [Mx, My, 2] (max, min; 1/s) and "stresses" [Mx, My, 3] (Pa)."""
        on_device = device or _is_device(mask)
        shape = self.shape
        m = _Buf(mask, shape)
        if m.device is not None and m.device != on_device:
            raise ValueError("mask and outputs must both be on the host or both on the device")
        want = {"edot": (edot, 2), "stresses": (stresses, 3)}
        out = {}
        for k, (on, d) in want.items():
            if not on:
                continue
            if on_device:
                import torch
                out[k] = torch.empty((*shape, d), dtype=torch.float64, device=f"cuda:{self.device}")
            else:
                out[k] = np.empty((*shape, d))
        bufs = {k: _Buf(v, v.shape) for k, v in out.items()}
        where = _capi.MEM_DEVICE if on_device else _capi.MEM_HOST
        self._check(self.lib.pism_gpu_ssa_strain_rates(self._h, m.ptr, bufs["edot"].ptr if "edot" in bufs else None,
                                                       bufs["stresses"].ptr if "stresses" in bufs else None, where),
                    "compute_2D_principal_strain_rates")
        return {k: (bufs[k].keep if on_device else out[k]) for k in out}

    def eigen_calving(self, dt: float, K: float, mask, Href, thickness) -> dict:
        """EigenCalving::update (PISMEigenCalving.cc:77-235) over dt seconds with constant K
        (m s) on the current velocity: returns the new "mask", "Href" and "thickness" (the
        caller's arrays are not changed).  Host arrays or CUDA tensors, all of one kind."""
        shape = self.shape
        kinds = {_is_device(a) for a in (mask, Href, thickness)}
        if len(kinds) != 1:
            raise ValueError("mask, Href and thickness must all be host arrays or all CUDA tensors")
        on_device = kinds.pop()
        # the library overwrites its arguments: hand it copies
        if on_device:
            import torch
            bufs = [_Buf(a.to(torch.float64).reshape(shape).clone(), shape) for a in (mask, Href, thickness)]
        else:
            bufs = [_Buf(np.array(a, dtype=np.float64).reshape(shape), shape) for a in (mask, Href, thickness)]
        where = _capi.MEM_DEVICE if on_device else _capi.MEM_HOST
        self._check(self.lib.pism_gpu_ssa_eigen_calving(self._h, float(dt), float(K), bufs[0].ptr, bufs[1].ptr,
                                                        bufs[2].ptr, where), "EigenCalving::update")
        return {k: b.keep for k, b in zip(("mask", "Href", "thickness"), bufs)}

    def eigen_calving_max_timestep(self, K: float, mask) -> dict:
        """EigenCalving::max_timestep (PISMEigenCalving.cc:249-341) on the current velocity:
        "dt" (s), "max_rate", "mean_rate" (m/s) and "count" of calving cells."""
        m = _Buf(mask, self.shape)
        res = (C.c_double * 4)()
        where = _capi.MEM_DEVICE if m.device else _capi.MEM_HOST
        self._check(self.lib.pism_gpu_ssa_eigen_calving_max_timestep(self._h, float(K), m.ptr, C.cast(res, _D), where),
                    "EigenCalving::max_timestep")
        return dict(zip(("dt", "max_rate", "mean_rate", "count"), list(res)))

    # ---- stage methods (one reference method each) ----
    def assemble_rhs(self):
        self._check(self.lib.pism_gpu_ssa_assemble_rhs(self._h), "assemble_rhs")

    def compute_hardav_staggered(self):
        self._check(self.lib.pism_gpu_ssa_compute_hardness(self._h), "compute_hardav_staggered")

    def compute_nuH_staggered(self, nuH_regularization: float):
        self._check(self.lib.pism_gpu_ssa_compute_nuH(self._h, nuH_regularization), "compute_nuH_staggered")

    def apply(self, x_dev, y_dev):
        """y = A x on device tensors ([Mx, My, 2] float64 CUDA)."""
        self._check(self.lib.pism_gpu_ssa_apply(self._h, C.c_void_p(x_dev.data_ptr()),
                                                C.c_void_p(y_dev.data_ptr())), "apply")

    def apply_preconditioner(self, r_dev, z_dev):
        """z = M^-1 r with the active preconditioner at the current nu*H / beta (PCApply);
        device tensors [Mx, My, 2] float64, not the same tensor."""
        self._check(self.lib.pism_gpu_ssa_apply_preconditioner(self._h, C.c_void_p(r_dev.data_ptr()),
                                                               C.c_void_p(z_dev.data_ptr())), "PCApply")

    def linear_solve_rhs(self, b_dev, x_dev):
        """A x = b for a device right-hand side b ([Mx, My, 2] float64 CUDA); x holds the initial
        guess and receives the solution.  Returns (iterations, relative residual)."""
        its = C.c_int(0)
        res = C.c_double(0)
        self._check(self.lib.pism_gpu_ssa_linear_solve_rhs(self._h, C.c_void_p(b_dev.data_ptr()),
                                                           C.c_void_p(x_dev.data_ptr()), C.byref(its), C.byref(res)),
                    "KSPSolve")
        return its.value, res.value

    def linear_solve(self, x_dev):
        its = C.c_int(0)
        res = C.c_double(0)
        self._check(self.lib.pism_gpu_ssa_linear_solve(self._h, C.c_void_p(x_dev.data_ptr()), C.byref(its),
                                                       C.byref(res)), "KSPSolve")
        return its.value, res.value


class _StrengthExtension:
    """SSAStrengthExtension (SSA.hh:39-58) of a solver: its parameters are configuration fields."""

    def __init__(self, ssa):
        self._ssa = ssa

    def set_min_thickness(self, thickness):
        self._ssa.set_config(self._ssa.config.copy(min_thickness_strength_extension_ssa=float(thickness)))

    def get_min_thickness(self):
        return self._ssa.config.min_thickness_strength_extension_ssa


SSAFD.strength_extension = property(lambda self: _StrengthExtension(self),
                                    doc="SSA::strength_extension (SSA.hh:111): its minimum thickness")


def SSAFD_GPUFactory(grid: GridDesc, config: SSAConfig | None = None) -> SSAFD:
    """The SSAFactory of this solver (typedef SSAFactory, SSA.hh:77; SSAFDFactory SSAFD.cc:47-49)."""
    return SSAFD(grid, config)


class StressBalance:
    """StressBalance (PISMStressBalance.hh) over this SSAFD with the ConstantInColumn modifier
    (SSB_Modifier.hh:71-74): update() runs the SSA solve and, unless fast, the 3-D fields
    its consumers read (PISMStressBalance.cc:79-116), all on the device; the getters return
    the last update's fields."""

    def __init__(self, ssa: SSAFD, device_outputs: bool = False):
        self.ssa = ssa
        self.device_outputs = device_outputs
        self._bmr = None
        self._fields = None

    def set_basal_melt_rate(self, bmr_input):
        """StressBalance::set_basal_melt_rate (PISMStressBalance.cc:73-76)."""
        self._bmr = bmr_input

    def set_boundary_conditions(self, locations, velocities):
        self.ssa.set_boundary_conditions(locations, velocities)

    def update(self, fast: bool = False, melange_back_pressure=None):
        """StressBalance::update (PISMStressBalance.cc:79-116)."""
        self.ssa.update(fast, melange_back_pressure)
        if not fast:
            self._fields = self.ssa.stress_balance_3d(self._bmr, device=self.device_outputs)

    def advective_velocity(self):
        return self.ssa.velocity()

    def basal_frictional_heating(self):
        return self.ssa.basal_frictional_heating()

    def _field(self, name):
        if self._fields is None:
            raise SSAError("StressBalance::update(fast=False) has not run")
        return self._fields[name]

    def velocity_u(self):
        return self._field("u")

    def velocity_v(self):
        return self._field("v")

    def velocity_w(self):
        return self._field("w")

    def volumetric_strain_heating(self):
        return self._field("strain_heating")

    def compute_2D_principal_strain_rates(self, mask=None):
        """ShallowStressBalance::compute_2D_principal_strain_rates (ShallowStressBalance.cc:224-305)
        of the advective velocity: [Mx, My, 2], (max, min) eigenvalue (1/s)."""
        return self.ssa.strain_rates(mask, edot=True, stresses=False, device=self.device_outputs)["edot"]

    def compute_2D_stresses(self, mask=None):
        """ShallowStressBalance::compute_2D_stresses (ShallowStressBalance.cc:308-386):
        [Mx, My, 3] deviatoric stresses (Pa)."""
        return self.ssa.strain_rates(mask, edot=False, stresses=True, device=self.device_outputs)["stresses"]


class EigenCalving:
    """calving::EigenCalving (PISMEigenCalving.hh) over a StressBalance: update() applies the
    eigen-calving step to the model's mask, Href and thickness in place (numpy arrays or CUDA
    tensors); max_timestep() returns the CFL time step, None unless cfl_eigen_calving."""

    def __init__(self, stress_balance: StressBalance, K: float = 0.0, restrict_timestep: bool = False):
        g = stress_balance.ssa.grid
        if abs(g.dx - g.dy) / min(g.dx, g.dy) > 1e-2:   # EigenCalving::init, PISMEigenCalving.cc:63-69
            raise SSAError("eigen_calving using a non-square grid cell is not implemented")
        self.stress_balance = stress_balance
        self.K = float(K)                         # eigen_calving_K (m s), pism_config.cdl:581-585
        self.restrict_timestep = restrict_timestep   # cfl_eigen_calving
        self.last_rates = None

    def update(self, dt, pism_mask, Href, ice_thickness):
        """EigenCalving::update(dt, pism_mask, Href, ice_thickness) (PISMEigenCalving.cc:77-235)."""
        out = self.stress_balance.ssa.eigen_calving(dt, self.K, pism_mask, Href, ice_thickness)
        for name, dst in (("mask", pism_mask), ("Href", Href), ("thickness", ice_thickness)):
            if _is_device(dst):
                dst.copy_(out[name].reshape(dst.shape))
            else:
                dst[...] = np.asarray(out[name]).reshape(dst.shape)

    def max_timestep(self, mask):
        """EigenCalving::max_timestep (PISMEigenCalving.cc:249-341) for the model's mask: the
        allowed time step in seconds, or None (no restriction) unless cfl_eigen_calving; the
        rates behind it are kept in last_rates."""
        if not self.restrict_timestep:
            return None
        self.last_rates = self.stress_balance.ssa.eigen_calving_max_timestep(self.K, mask)
        return self.last_rates["dt"]


class SSAFEMFailure(SSAError):
    """SSAFEM::solve's "SSAFEM solve failed to converge" (SSAFEM.cc:179-183)."""


class SSAFEM(SSAFD):
    """pism::stressbalance::SSAFEM (SSAFEM.hh) on the B200: the Q1 finite-element SSA, with the
    inputs, boundary conditions, initial guess and getters of SSAFD; solve() runs Newton on
    the weak form from the current velocity (SSAFEM::solve, SSAFEM.cc:170-232).  The
    nonlinear and linear settings are `options` (pism_gpu_ssafem_options)."""

    def __init__(self, grid: GridDesc, config: SSAConfig | None = None, device: int = 0, **options):
        super().__init__(grid, config, device)
        self.options = CFemOptions()
        self.lib.pism_gpu_ssafem_options_defaults(C.byref(self.options))
        self.options.icefree_thickness = self.config.mask_icefree_thickness_standard
        self.options.is_floating_thickness = self.config.mask_is_floating_thickness_standard
        for k, v in options.items():
            setattr(self.options, k, v)
        self._fem_stats = CFemStats()

    def solve(self, out=None):
        """SSAFEM::solve; returns the velocity ([Mx, My, 2])."""
        rc = self.lib.pism_gpu_ssafem_solve(self._h, C.byref(self.options), C.byref(self._fem_stats))
        if rc == _capi.EPICARD:
            msg = self.lib.pism_gpu_ssa_last_error(self._h).decode()
            raise SSAFEMFailure(f"SSAFEM solve failed to converge: {msg}")
        self._check(rc, "SSAFEM::solve")
        return self.velocity(out)

    def stats(self) -> dict:
        return self._fem_stats.as_dict()


def SSAFEMFactory(grid: GridDesc, config: SSAConfig | None = None) -> SSAFEM:
    """The SSAFactory of the finite-element solver (SSAFEMFactory, SSAFEM.cc:105-107)."""
    return SSAFEM(grid, config)
