"""CPU restatement of PISM's SSAFEM (src/base/stressbalance/ssa/SSAFEM.cc:151-840,
FETools.cc / FETools.hh) — TEST INFRASTRUCTURE ONLY: the checker of the GPU Q1 finite-element
SSA, never the thing measured or shipped.

Q1 elements between grid nodes, 2 x 2 Gauss quadrature (FETools.cc:512-519), the coefficients
cached at the quadrature points (SSAFEM::cacheQuadPtValues, SSAFEM.cc:233-375), the weak-form
residual (compute_local_function, SSAFEM.cc:441-532) and its Newton Jacobian
(compute_local_jacobian, SSAFEM.cc:571-700) with Dirichlet rows of scale x (u - u_bc)
(DirichletData_Vector, FETools.cc:671-741).  The reference solves F(u) = 0 with PETSc's SNES
(Newton with a line search; PETSc is a third-party dependency absent from the reference tree);
here Newton steps use a direct sparse solve and a backtracking line search, run to a tighter
residual than SNES's default, so the answer is the discrete solution itself.  Pinned by the
reference's SSAFEM regression tables (test I, test J, the linear and plug flows).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import ssafd_oracle as O

GAUSS = 0.57735026918962573                                           # FETools.cc:512-516
QUAD_POINTS = ((-GAUSS, -GAUSS), (GAUSS, -GAUSS), (GAUSS, GAUSS), (-GAUSS, GAUSS))
NODE_OFFSETS = ((0, 0), (1, 0), (1, 1), (0, 1))                        # DOFMap, FETools.cc:206-207
DIRICHLET_SCALE = 1.0e9                                                # SSAFEM::init_impl, SSAFEM.cc:128-131


def shape(k, x, y):
    """ShapeQ1::shape0..3, FETools.hh:187-213: (value, d/dx, d/dy) on the reference square."""
    if k == 0:
        return (1 - x) * (1 - y) / 4., -(1 - y) / 4., -(1 - x) / 4
    if k == 1:
        return (1 + x) * (1 - y) / 4., (1 - y) / 4., -(1 + x) / 4
    if k == 2:
        return (1 + x) * (1 + y) / 4., (1 + y) / 4., (1 + x) / 4
    return (1 - x) * (1 + y) / 4., -(1 + y) / 4., (1 - x) / 4


def germs(dx, dy):
    """Quadrature::Quadrature, FETools.cc:300-316: test-function values and derivatives at the
    quadrature points (val, gx, gy: [q][k]) and the weighted Jacobian JxW[q]."""
    jx, jy = 0.5 * dx, 0.5 * dy
    val, gx, gy = np.zeros((4, 4)), np.zeros((4, 4)), np.zeros((4, 4))
    for q, (xq, yq) in enumerate(QUAD_POINTS):
        for k in range(4):
            v, ddx, ddy = shape(k, xq, yq)
            val[q, k], gx[q, k], gy[q, k] = v, ddx / jx, ddy / jy
    return val, gx, gy, np.full(4, jx * jy * 1.0)


class Elements:
    """ElementMap (FETools.cc:38-83) for one process: the elements whose lower-left node is
    (ei, ej); Mx of them along a periodic direction, Mx - 1 otherwise; and the four node
    indices of each, [4, nex, ney] (k order of DOFMap)."""

    def __init__(self, grid: O.Grid):
        self.grid = grid
        self.nex = grid.Mx if grid.periodicity & O.X_PERIODIC else grid.Mx - 1
        self.ney = grid.My if grid.periodicity & O.Y_PERIODIC else grid.My - 1
        ei, ej = np.meshgrid(np.arange(self.nex), np.arange(self.ney), indexing="ij")
        self.ni = np.stack([(ei + di) % grid.Mx for di, _ in NODE_OFFSETS])
        self.nj = np.stack([(ej + dj) % grid.My for _, dj in NODE_OFFSETS])
        self.node = self.ni * grid.My + self.nj   # flat node index

    def local(self, field):
        """the element-local values of a node field [Mx, My, ...] -> [4, nex, ney, ...]"""
        return field[self.ni, self.nj]


def quadrature_coefficients(grid: O.Grid, cfg: O.Config, inp: O.Inputs, el: Elements):
    """SSAFEM::cacheQuadPtValues, SSAFEM.cc:233-375: H, b, tau_c, the driving stress
    -rho g H grad(s) and the GeometryCalculator mask at each quadrature point, and the hardness
    averaged over the column of enthalpy interpolated to the quadrature point."""
    val, gx, gy, _ = germs(grid.dx, grid.dy)

    def at_q(field, w):
        loc = el.local(np.asarray(field, dtype=np.float64))
        out = np.zeros((4,) + loc.shape[1:])
        for q in range(4):
            for k in range(4):
                out[q] = out[q] + w[q, k] * loc[k]
        return out

    H, b, tauc = at_q(inp.thickness, val), at_q(inp.bed, val), at_q(inp.tauc, val)
    hx, hy = at_q(inp.surface, gx), at_q(inp.surface, gy)
    taud_u = -cfg.ice_density * cfg.standard_gravity * H * hx
    taud_v = -cfg.ice_density * cfg.standard_gravity * H * hy
    mask, _ = O.geometry_mask_surface(cfg, b, H)
    if cfg.flow_law != "isothermal_glen" and inp.enthalpy is None:
        raise ValueError(f"the flow law {cfg.flow_law} needs enthalpy")
    if cfg.flow_law == "isothermal_glen":
        B = O.averaged_hardness(cfg, H.ravel(), None, None).reshape(H.shape)
    else:
        E = np.asarray(inp.enthalpy, dtype=np.float64)
        Eq = at_q(E, val)   # [4, nex, ney, Mz]
        B = O.averaged_hardness(cfg, H.ravel(), np.asarray(grid.z), Eq.reshape(-1, E.shape[-1])).reshape(H.shape)
    return {"H": H, "b": b, "tauc": tauc, "taud_u": taud_u, "taud_v": taud_v, "mask": O.as_int(mask), "B": B}


def nuH_and_beta(cfg: O.Config, C, u, v, Du):
    """SSAFEM::PointwiseNuHAndBeta, SSAFEM.cc:393-432, with FlowLaw::effective_viscosity
    (flowlaws.hh:100-112) and drag_with_derivative (basal_resistance.cc:59-68, 174-190):
    (eta, deta/dgamma, beta, dbeta/d(|u|^2 / 2))."""
    n = cfg.ssa_Glen_exponent
    power = (1.0 - n) / (2.0 * n)
    gamma = 0.5 * (Du[0] * Du[0] + Du[1] * Du[1] + (Du[0] + Du[1]) * (Du[0] + Du[1]) + 2 * Du[2] * Du[2])
    nu = 0.5 * C["B"] * np.power(O.schoof_reg(cfg) + gamma, power)
    dnu = power * nu / (O.schoof_reg(cfg) + gamma)
    thin = C["H"] < cfg.min_thickness_strength_extension_ssa
    eta = np.where(thin, O.notional_strength(cfg), cfg.epsilon_ssa + nu * C["H"])
    deta = np.where(thin, 0.0, dnu * C["H"])
    magreg2 = cfg.plastic_regularization ** 2 + u * u + v * v
    if not cfg.do_pseudo_plastic_till:
        drag = C["tauc"] / np.sqrt(magreg2)
        ddrag = -1 * drag / magreg2
    else:
        qq = cfg.pseudo_plastic_q
        if cfg.sliding_scale_factor_reduces_tauc > 0.0:
            Aq = cfg.sliding_scale_factor_reduces_tauc ** qq
            drag = (C["tauc"] / Aq) * np.power(magreg2, 0.5 * (qq - 1)) * cfg.pseudo_plastic_uthreshold ** (-qq)
        else:
            drag = C["tauc"] * np.power(magreg2, 0.5 * (qq - 1)) * cfg.pseudo_plastic_uthreshold ** (-qq)
        ddrag = (qq - 1) * drag / magreg2
    M = C["mask"]
    grounded_ice = O.m_grounded_ice(M)
    beta = np.where(grounded_ice, drag, np.where(O.m_ice_free_land(M), cfg.beta_ice_free_bedrock, 0.0))
    dbeta = np.where(grounded_ice, ddrag, 0.0)
    return eta, deta, beta, dbeta


class SSAFEMOracle:
    """The discrete SSAFEM problem of one set of inputs: residual, Jacobian and a Newton
    solve.  Dirichlet data apply where bc_mask > 0.5 when bc_mask and bc_values are given
    (SSA::set_boundary_conditions)."""

    def __init__(self, grid: O.Grid, cfg: O.Config, inp: O.Inputs, dirichlet_scale=DIRICHLET_SCALE):
        self.grid, self.cfg, self.inp = grid, cfg, inp
        self.el = Elements(grid)
        self.C = quadrature_coefficients(grid, cfg, inp, self.el)
        self.val, self.gx, self.gy, self.JxW = germs(grid.dx, grid.dy)
        self.scale = dirichlet_scale
        shape2 = (grid.Mx, grid.My)
        if inp.bc_mask is not None and inp.bc_values is not None:
            self.bc = np.asarray(inp.bc_mask, dtype=np.float64) > 0.5
            self.bcv = np.asarray(inp.bc_values, dtype=np.float64)
        else:
            self.bc = np.zeros(shape2, dtype=bool)
            self.bcv = np.zeros(shape2 + (2,))

    def _local_velocity(self, vel):
        """element-local velocities with Dirichlet values at Dirichlet nodes (DirichletData::update)"""
        w = np.where(self.bc[..., None], self.bcv, vel)
        return self.el.local(w)   # [4, nex, ney, 2]

    def _quadrature_values(self, loc):
        u, v = np.zeros((4,) + loc.shape[1:3]), np.zeros((4,) + loc.shape[1:3])
        Du = np.zeros((4, 3) + loc.shape[1:3])
        for q in range(4):
            for k in range(4):
                u[q] = u[q] + self.val[q, k] * loc[k, ..., 0]
                v[q] = v[q] + self.val[q, k] * loc[k, ..., 1]
                Du[q, 0] = Du[q, 0] + self.gx[q, k] * loc[k, ..., 0]
                Du[q, 1] = Du[q, 1] + self.gy[q, k] * loc[k, ..., 1]
                Du[q, 2] = Du[q, 2] + 0.5 * (self.gy[q, k] * loc[k, ..., 0] + self.gx[q, k] * loc[k, ..., 1])
        return u, v, Du

    def residual(self, vel):
        """compute_local_function, SSAFEM.cc:441-532: [Mx, My, 2]."""
        g, C = self.grid, self.C
        loc = self._local_velocity(vel)
        u, v, Du = self._quadrature_values(loc)
        r = np.zeros((4,) + loc.shape[1:3] + (2,))
        for q in range(4):
            Cq = {k: a[q] for k, a in C.items()}
            eta, _, beta, _ = nuH_and_beta(self.cfg, Cq, u[q], v[q], Du[q])
            tbu, tbv = u[q] * (-beta), v[q] * (-beta)
            Ux, Vy, UyVx = Du[q, 0], Du[q, 1], 2.0 * Du[q, 2]
            for k in range(4):
                px, py, pv = self.gx[q, k], self.gy[q, k], self.val[q, k]
                r[k, ..., 0] += self.JxW[q] * (eta * (px * (4.0 * Ux + 2.0 * Vy) + py * UyVx)
                                               - pv * (tbu + C["taud_u"][q]))
                r[k, ..., 1] += self.JxW[q] * (eta * (px * UyVx + py * (2.0 * Ux + 4.0 * Vy))
                                               - pv * (tbv + C["taud_v"][q]))
        F = np.zeros((g.Mx * g.My, 2))
        for k in range(4):
            np.add.at(F, self.el.node[k].ravel(), r[k].reshape(-1, 2))
        F = F.reshape(g.Mx, g.My, 2)
        return np.where(self.bc[..., None], self.scale * (vel - self.bcv), F)

    def jacobian(self, vel):
        """compute_local_jacobian, SSAFEM.cc:571-700, as a sparse (2 Mx My)^2 matrix; unknowns
        ordered (node, component), node = i My + j."""
        g, C = self.grid, self.C
        loc = self._local_velocity(vel)
        u, v, Du = self._quadrature_values(loc)
        K = np.zeros((8, 8) + loc.shape[1:3])
        for q in range(4):
            Cq = {k: a[q] for k, a in C.items()}
            eta, deta, beta, dbeta = nuH_and_beta(self.cfg, Cq, u[q], v[q], Du[q])
            jw = self.JxW[q]
            U, V = u[q], v[q]
            Ux, Vy, UyVx = Du[q, 0], Du[q, 1], 2.0 * Du[q, 2]
            for l in range(4):
                phi, phx, phy = self.val[q, l], self.gx[q, l], self.gy[q, l]
                gamma_u = (2.0 * Ux + Vy) * phx + Du[q, 2] * phy
                gamma_v = Du[q, 2] * phx + (Ux + 2.0 * Vy) * phy
                eta_u, eta_v = deta * gamma_u, deta * gamma_v
                taub_xu = -dbeta * U * U * phi - beta * phi
                taub_xv = -dbeta * U * V * phi
                taub_yu = -dbeta * V * U * phi
                taub_yv = -dbeta * V * V * phi - beta * phi
                for k in range(4):
                    psi, psx, psy = self.val[q, k], self.gx[q, k], self.gy[q, k]
                    K[k * 2 + 0, l * 2 + 0] += jw * (eta_u * (psx * (4 * Ux + 2 * Vy) + psy * UyVx)
                                                     + eta * (4 * psx * phx + psy * phy) - psi * taub_xu)
                    K[k * 2 + 0, l * 2 + 1] += jw * (eta_v * (psx * (4 * Ux + 2 * Vy) + psy * UyVx)
                                                     + eta * (2 * psx * phy + psy * phx) - psi * taub_xv)
                    K[k * 2 + 1, l * 2 + 0] += jw * (eta_u * (psx * UyVx + psy * (2 * Ux + 4 * Vy))
                                                     + eta * (psx * phy + 2 * psy * phx) - psi * taub_yu)
                    K[k * 2 + 1, l * 2 + 1] += jw * (eta_v * (psx * UyVx + psy * (2 * Ux + 4 * Vy))
                                                     + eta * (psx * phx + 4 * psy * phy) - psi * taub_yv)
        bc_flat = self.bc.ravel()
        rows, cols, vals = [], [], []
        for k in range(4):
            nk = self.el.node[k].ravel()
            for l in range(4):
                nl = self.el.node[l].ravel()
                keep = ~bc_flat[nk] & ~bc_flat[nl]
                for c in range(2):
                    for d in range(2):
                        rows.append(2 * nk[keep] + c)
                        cols.append(2 * nl[keep] + d)
                        vals.append(K[k * 2 + c, l * 2 + d].ravel()[keep])
        dofs = np.nonzero(bc_flat)[0]
        for c in range(2):
            rows.append(2 * dofs + c)
            cols.append(2 * dofs + c)
            vals.append(np.full(len(dofs), self.scale))
        n = 2 * g.Mx * g.My
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))

    def solve(self, vel0=None, rtol=1e-11, stol=1e-13, maxit=100):
        """Newton with a backtracking line search on ||F|| until ||F|| <= rtol ||F(u0)|| or
        a step changes the velocity by less than stol of its norm (the residual then sits at
        its rounding floor).  Returns the velocity [Mx, My, 2] and the number of Newton steps."""
        g = self.grid
        vel = np.zeros((g.Mx, g.My, 2)) if vel0 is None else np.array(vel0, dtype=np.float64)
        F = self.residual(vel)
        f0 = fn = np.linalg.norm(F)
        its = 0
        while fn > rtol * f0 and its < maxit:
            J = self.jacobian(vel)
            du = spla.spsolve(J.tocsc(), -F.reshape(-1)).reshape(vel.shape)
            lam = 1.0
            while True:
                trial = vel + lam * du
                Ft = self.residual(trial)
                ft = np.linalg.norm(Ft)
                if ft < (1.0 - 1e-4 * lam) * fn or lam < 1e-6:
                    break
                lam *= 0.5
            small = np.linalg.norm(lam * du) <= stol * np.linalg.norm(trial)
            vel, F, fn = trial, Ft, ft
            its += 1
            if small:
                break
        return vel, its
