// ssa_kernels.cu — sm_100a kernels of the B200 SSAFD solver.
//
// Every kernel restates one piece of the reference's SSAFD arithmetic (file:line
// in each comment).  All are HBM-bound stencil / vector kernels: cells are mapped
// to 32 (j, contiguous) x 8 (i) tiles so that a warp reads 32 consecutive double2
// values (512 B) and the i +- 1 rows of the stencil are re-read from L1 by the
// neighbouring warps of the same block; blocks loop over tiles (grid = a multiple
// of the SM count).  Reductions are fused into the producing kernel: each block
// writes its partial sums, and the last block to finish (atomic ticket) adds them
// in block order — deterministic — and updates the solver scalars on the device,
// so no kernel boundary or host round trip is spent on a dot product.
#include <cstdio>

#include "ssa_internal.h"
#include "ssa_stencil.cuh"
#include "ssa_reduce.cuh"

namespace pism_gpu {

constexpr int TJ = 32;  // tile width along j (contiguous)
constexpr int TI = 8;   // tile height along i
constexpr int NT = TJ * TI;

struct TileMap {
  int tiles_j, tiles;
  __device__ __forceinline__ bool cell_of(const GridDev &g, int t, int &i, int &j) const {
    int ti = t / tiles_j, tj = t - ti * tiles_j;
    j = tj * TJ + (threadIdx.x & (TJ - 1));
    i = ti * TI + (threadIdx.x >> 5);
    return i < g.Mx && j < g.My;
  }
};

static TileMap make_tiles(const GridDev &g) {
  TileMap m;
  m.tiles_j = (g.My + TJ - 1) / TJ;
  m.tiles = m.tiles_j * ((g.Mx + TI - 1) / TI);
  return m;
}

// ---------------------------------------------------------------------------
// input conversion: masks stored as doubles -> integers (IceModelVec2Int::as_int,
// IceModelVec_inline.hh:94-100)
// ---------------------------------------------------------------------------
__global__ void k_convert_masks(int N, const double *mask, const double *bc_mask, int8_t *mask_i,
                                uint8_t *bc_i) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    mask_i[k] = (int8_t)(int)floor(mask[k] + 0.5);
    bc_i[k] = bc_mask ? (uint8_t)((int)floor(bc_mask[k] + 0.5) == 1) : (uint8_t)0;
  }
}

// ---------------------------------------------------------------------------
// driving stress + right-hand side + stencil flags (once per solve)
//   SSA::compute_driving_stress  SSA.cc:211-353
//   SSAFD::assemble_rhs          SSAFD.cc:282-417
//   SSAFD::is_marginal           SSAFD.cc:1657-1682, CFBC weights SSAFD.cc:594-684
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) k_prepare(GridDev g, TileMap tm, pism_gpu_ssa_config c, int periodicity,
                                                const double *__restrict__ H, const double *__restrict__ srf,
                                                const double *__restrict__ bed, const int8_t *__restrict__ mask,
                                                const uint8_t *__restrict__ bc, const double2 *__restrict__ bcv,
                                                const double *__restrict__ melange, double2 *__restrict__ taud,
                                                double2 *__restrict__ rhs, uint32_t *__restrict__ flags) {
  const double dx = g.dx, dy = g.dy;
  const bool cfbc = c.calving_front_stress_boundary_condition != 0;
  const bool bb = c.ssa_dirichlet_bc != 0;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j;
    if (!tm.cell_of(g, t, i, j)) continue;
    const int k = cell(g, i, j);
    const int kE = nbr(g, i, j, 1, 0), kW = nbr(g, i, j, -1, 0), kN = nbr(g, i, j, 0, 1), kS = nbr(g, i, j, 0, -1);
    const int M = mask[k], Me = mask[kE], Mw = mask[kW], Mn = mask[kN], Ms = mask[kS];
    const int Mne = mask[nbr(g, i, j, 1, 1)], Mse = mask[nbr(g, i, j, 1, -1)], Mnw = mask[nbr(g, i, j, -1, 1)],
              Msw = mask[nbr(g, i, j, -1, -1)];
    const double Hc = H[k];

    // ---- driving stress (SSA.cc:234-352) ----
    const double n = c.ssa_Glen_exponent;
    const double pressure = ec_pressure(c, Hc);
    double2 td = make_double2(0.0, 0.0);
    if (pressure > 0.0) {
      double h_x = 0.0, h_y = 0.0;
      if (m_grounded(M) && c.surface_gradient_eta) {
        const double etapow = (2.0 * n + 2.0) / n, invpow = 1.0 / etapow, dinvpow = (-n - 2.0) / (2.0 * n + 2.0);
        const double minThickEtaTransform = 5.0;
        if (Hc > 0.0) {
          const double myH = (Hc < minThickEtaTransform ? minThickEtaTransform : Hc);
          const double eta = pow(myH, etapow), factor = invpow * pow(eta, dinvpow);
          h_x = factor * (pow(H[kE], etapow) - pow(H[kW], etapow)) / (2 * dx);
          h_y = factor * (pow(H[kN], etapow) - pow(H[kS], etapow)) / (2 * dy);
        }
        h_x += (bed[kE] - bed[kW]) / (2 * dx);
        h_y += (bed[kN] - bed[kS]) / (2 * dy);
      } else if (c.compute_surf_grad_inward_ssa) {
        // IceModelVec2S::diff_x_p / diff_y_p (iceModelVec2.cc:501-530)
        if ((periodicity & PISM_X_PERIODIC) || (i != 0 && i != g.Mx - 1))
          h_x = (srf[kE] - srf[kW]) / (2 * dx);
        else if (i == 0)
          h_x = (srf[kE] - srf[k]) / dx;
        else
          h_x = (srf[k] - srf[kW]) / dx;
        if ((periodicity & PISM_Y_PERIODIC) || (j != 0 && j != g.My - 1))
          h_y = (srf[kN] - srf[kS]) / (2 * dy);
        else if (j == 0)
          h_y = (srf[kN] - srf[k]) / dy;
        else
          h_y = (srf[k] - srf[kS]) / dy;
      } else {
        double west = 1, east = 1, south = 1, north = 1;
        if ((m_grounded(M) && m_floating_ice(Me)) || (m_floating_ice(M) && m_grounded(Me)) ||
            (m_floating_ice(M) && m_ice_free_ocean(Me)))
          east = 0;
        if ((m_grounded(M) && m_floating_ice(Mw)) || (m_floating_ice(M) && m_grounded(Mw)) ||
            (m_floating_ice(M) && m_ice_free_ocean(Mw)))
          west = 0;
        if ((m_grounded(M) && m_floating_ice(Mn)) || (m_floating_ice(M) && m_grounded(Mn)) ||
            (m_floating_ice(M) && m_ice_free_ocean(Mn)))
          north = 0;
        if ((m_grounded(M) && m_floating_ice(Ms)) || (m_floating_ice(M) && m_grounded(Ms)) ||
            (m_floating_ice(M) && m_ice_free_ocean(Ms)))
          south = 0;
        if (cfbc) {
          if (m_icy(M) && m_ice_free(Me)) east = 0;
          if (m_icy(M) && m_ice_free(Mw)) west = 0;
          if (m_icy(M) && m_ice_free(Mn)) north = 0;
          if (m_icy(M) && m_ice_free(Ms)) south = 0;
        }
        const double s0 = srf[k];
        if (east + west > 0)
          h_x = 1.0 / (west + east) * (west * ((s0 - srf[kW]) / dx) + east * ((srf[kE] - s0) / dx));
        if (north + south > 0)
          h_y = 1.0 / (south + north) * (south * ((s0 - srf[kS]) / dy) + north * ((srf[kN] - s0) / dy));
      }
      td.x = -pressure * h_x;
      td.y = -pressure * h_y;
    }
    taud[k] = td;

    // ---- flags and right-hand side ----
    const bool is_bc = bc[k] != 0;
    uint32_t f = F_WEIGHTS | ((uint32_t)(M & 7) << F_MASK_SHIFT);
    double2 b = td;
    if (cfbc) {
      bool marginal;
      if (bb)
        marginal = m_icy(M) && (m_ice_free(Me) || m_ice_free(Mw) || m_ice_free(Mn) || m_ice_free(Ms) ||
                                m_ice_free(Mne) || m_ice_free(Mse) || m_ice_free(Mnw) || m_ice_free(Msw));
      else
        marginal = m_icy(M) && (m_ice_free_ocean(Me) || m_ice_free_ocean(Mw) || m_ice_free_ocean(Mn) ||
                                m_ice_free_ocean(Ms) || m_ice_free_ocean(Mne) || m_ice_free_ocean(Mse) ||
                                m_ice_free_ocean(Mnw) || m_ice_free_ocean(Msw));
      if (m_ice_free(M)) {
        f |= F_DIAG_ONLY;
        b = make_double2(0.0, 0.0);   // m_scaling * ice_free_default_velocity (= 0)
      } else if (marginal) {
        auto fr = [&](int Mq) { return bb ? m_ice_free_ocean(Mq) : m_ice_free(Mq); };
        const bool e = fr(Me), w = fr(Mw), nn = fr(Mn), s = fr(Ms), ne = fr(Mne), se = fr(Mse), nw = fr(Mnw),
                   sw = fr(Msw);
        if (e) f &= ~F_aPP;
        if (w) f &= ~F_aMM;
        if (nn) f &= ~F_bPP;
        if (s) f &= ~F_bMM;
        if (nn || ne) f &= ~F_aPn;
        if (e || ne) f &= ~F_bPe;
        if (e || se) f &= ~F_bMe;
        if (s || se) f &= ~F_aPs;
        if (s || sw) f &= ~F_aMs;
        if (w || sw) f &= ~F_bMw;
        if (w || nw) f &= ~F_bPw;
        if (nn || nw) f &= ~F_aMn;
        // ocean pressure imbalance (SSAFD.cc:370-403)
        const double H2 = Hc * Hc, bcell = bed[k], rho_g = c.ice_density * c.standard_gravity;
        double op;
        if (m_ocean(M))
          op = 0.5 * rho_g * (1.0 - (c.ice_density / c.sea_water_density)) * H2;
        else if (bcell >= c.sea_level)
          op = 0.5 * rho_g * H2;
        else
          op = 0.5 * rho_g * (H2 - (c.sea_water_density / c.ice_density) * pow(c.sea_level - bcell, 2.0));
        if (melange) op *= (1.0 - melange[k]);
        const int aMM = w ? 0 : 1, aPP = e ? 0 : 1, bMM = s ? 0 : 1, bPP = nn ? 0 : 1;
        b.x = td.x + (aMM - aPP) * op / dx;
        b.y = td.y + (bMM - bPP) * op / dy;
      }
    }
    if (c.nu_bedrock_set && Hc > 0.0) {   // HminFrozen = 0 (SSAFD.cc:535, 571-584)
      const double s0 = srf[k];
      if (bed[kW] > s0 && m_ice_free_land(Mw)) f |= F_NB_W;
      if (bed[kE] > s0 && m_ice_free_land(Me)) f |= F_NB_E;
      if (bed[kN] > s0 && m_ice_free_land(Mn)) f |= F_NB_N;
      if (bed[kS] > s0 && m_ice_free_land(Ms)) f |= F_NB_S;
    }
    if (is_bc) {
      f |= F_DIAG_ONLY | F_BC;
      const double2 v = bcv[k];
      b = make_double2(1.0e9 * v.x, 1.0e9 * v.y);
    }
    rhs[k] = b;
    flags[k] = f;
  }
}

// ---------------------------------------------------------------------------
// staggered vertically averaged hardness (SSAFD::compute_hardav_staggered,
// SSAFD.cc:1192-1246; FlowLaw::averaged_hardness, flowlaws.cc:141-185;
// fracture_induced_softening, SSAFD.cc:1282-1310)
// ---------------------------------------------------------------------------
__device__ double averaged_hardness(const pism_gpu_ssa_config &c, double thickness, int kb, const double *z,
                                    const double *E0, const double *E1) {
  double B = 0;
  if (kb > 0) {
    double h0 = hardness_parameter(c, 0.5 * (E0[0] + E1[0]), ec_pressure(c, thickness));
    for (int q = 1; q <= kb; ++q) {
      double h1 = hardness_parameter(c, 0.5 * (E0[q] + E1[q]), ec_pressure(c, thickness - z[q]));
      B += (z[q] - z[q - 1]) * (h0 + h1);
      h0 = h1;
    }
  }
  B *= 0.5;
  double depth = thickness - z[kb];
  B += depth * hardness_parameter(c, 0.5 * (E0[kb] + E1[kb]), ec_pressure(c, depth));
  return thickness > 0 ? B / thickness : 0.0;
}

__global__ void k_hardness(GridDev g, int N, pism_gpu_ssa_config c, const double *__restrict__ H,
                           const int8_t *__restrict__ mask, const double *__restrict__ enthalpy, int Mz,
                           const double *__restrict__ z, const double *__restrict__ fracture,
                           double2 *__restrict__ hardness) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int i = k / g.My, j = k - i * g.My;
    double out[2];
    for (int o = 0; o < 2; ++o) {
      const int oi = 1 - o, oj = o;
      const int kn = nbr(g, i, j, oi, oj);
      const bool ic = m_icy(mask[k]), in = m_icy(mask[kn]);
      double Hf;
      if (ic && in)
        Hf = 0.5 * (H[k] + H[kn]);
      else if (ic)
        Hf = H[k];
      else
        Hf = H[kn];
      if (Hf == 0) {
        out[o] = -1e6;
        continue;
      }
      if (c.flow_law == PISM_FLOW_LAW_ISOTHERMAL_GLEN) {
        out[o] = pow(c.ice_softness, -1.0 / c.ssa_Glen_exponent);   // flowlaws.cc:239-240
      } else {
        // IceGrid::kBelowHeight: largest q in [0, Mz-2] with z[q] <= Hf (gsl_interp_accel_find)
        int lo = 0, hi = Mz - 1;
        while (hi > lo + 1) {
          int mid = (lo + hi) / 2;
          if (z[mid] > Hf) hi = mid; else lo = mid;
        }
        out[o] = averaged_hardness(c, Hf, lo, z, enthalpy + (size_t)k * Mz, enthalpy + (size_t)kn * Mz);
      }
    }
    if (c.do_fracture_density && fracture) {
      const double n = c.ssa_Glen_exponent, eps = c.fracture_density_softening_lower_limit;
      for (int o = 0; o < 2; ++o) {
        const int kn = nbr(g, i, j, 1 - o, o);
        const double phi = 0.5 * (fracture[k] + fracture[kn]);
        const double soft = pow((1.0 - (1.0 - eps) * phi), -n);
        out[o] *= pow(soft, -1.0 / n);
      }
    }
    hardness[k] = make_double2(out[0], out[1]);
  }
}

// ---------------------------------------------------------------------------
// nu*H on the staggered grid, beta, under-relaxation and the L1 norms — fused.
//   SSAFD::compute_nuH_staggered       SSAFD.cc:1359-1421
//   SSAFD::compute_nuH_staggered_cfbc  SSAFD.cc:1441-1582 (m_work recomputed on the fly)
//   under-relaxation                   SSAFD.cc:1061-1064
//   SSAFD::compute_nuH_norm            SSAFD.cc:1170-1189 (L1 over the ghosted local
//                                      vectors: interior + one periodic ghost ring)
//   basal drag of the next assembly    SSAFD.cc:744-759
// ---------------------------------------------------------------------------
struct NuHParams {
  double reg, underrelax, Hmin, notional, schoof_reg, visc_power, enh_scaling, B_area;
  int with_norm;
};

struct WorkVal {  // one entry of the reference's m_work: derivative pair + weight
  double u, v, w;
};

template <bool CFBC>
__global__ void __launch_bounds__(NT) k_nuH(GridDev g, TileMap tm, pism_gpu_ssa_config c, NuHParams p,
                                            const double2 *__restrict__ vel, const double *__restrict__ H,
                                            const double2 *__restrict__ hardness, const int8_t *__restrict__ mask,
                                            const double *__restrict__ tauc, const double *__restrict__ gl_mask,
                                            double2 *__restrict__ nuH, double *__restrict__ beta,
                                            double *partials, unsigned *ticket, double *norm_out) {
  const double dx = g.dx, dy = g.dy;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j;
    if (!tm.cell_of(g, t, i, j)) continue;
    const int k = cell(g, i, j);
    const int kE = nbr(g, i, j, 1, 0), kN = nbr(g, i, j, 0, 1), kS = nbr(g, i, j, 0, -1), kW = nbr(g, i, j, -1, 0);
    const int kNE = nbr(g, i, j, 1, 1), kSE = nbr(g, i, j, 1, -1), kNW = nbr(g, i, j, -1, 1);
    const double2 uc = vel[k], ue = vel[kE], un = vel[kN], us = vel[kS], uw = vel[kW], une = vel[kNE],
                  use = vel[kSE], unw = vel[kNW];
    const double Hc = H[k], He = H[kE], Hn = H[kN];
    const double2 B = hardness[k];
    double r0, r1;
    if (!CFBC) {
      // east face (o = 0)
      double Hf = 0.5 * (Hc + He);
      if (Hf < p.Hmin) {
        r0 = p.notional;
      } else {
        double u_x = (ue.x - uc.x) / dx, u_y = (un.x + une.x - us.x - use.x) / (4 * dy);
        double v_x = (ue.y - uc.y) / dx, v_y = (un.y + une.y - us.y - use.y) / (4 * dy);
        double nu = 0.5 * B.x * pow(p.schoof_reg + second_invariant_2d(u_x, u_y, v_x, v_y), p.visc_power);
        r0 = nu * Hf;
        r0 *= p.enh_scaling;
        r0 += p.reg;
      }
      // north face (o = 1)
      Hf = 0.5 * (Hc + Hn);
      if (Hf < p.Hmin) {
        r1 = p.notional;
      } else {
        double u_x = (ue.x + une.x - uw.x - unw.x) / (4 * dx), u_y = (un.x - uc.x) / dy;
        double v_x = (ue.y + une.y - uw.y - unw.y) / (4 * dx), v_y = (un.y - uc.y) / dy;
        double nu = 0.5 * B.y * pow(p.schoof_reg + second_invariant_2d(u_x, u_y, v_x, v_y), p.visc_power);
        r1 = nu * Hf;
        r1 *= p.enh_scaling;
        r1 += p.reg;
      }
    } else {
      const int Mc = mask[k], Me = mask[kE], Mn = mask[kN], Ms = mask[kS], Mw = mask[kW], Mse = mask[kSE],
                Mnw = mask[kNW], Mne = mask[kNE];
      const bool ic = m_icy(Mc), ie = m_icy(Me), in = m_icy(Mn), is = m_icy(Ms), iw = m_icy(Mw), ise = m_icy(Mse),
                 inw = m_icy(Mnw), ine = m_icy(Mne);
      // m_work entries (SSAFD.cc:1463-1491), W_I at (a) between a and a+1 in i, W_J in j
      auto WI = [&](bool a, bool b, double2 va, double2 vb) {
        return (a && b) ? WorkVal{(vb.x - va.x) / dx, (vb.y - va.y) / dx, 1.0} : WorkVal{0.0, 0.0, 0.0};
      };
      auto WJ = [&](bool a, bool b, double2 va, double2 vb) {
        return (a && b) ? WorkVal{(vb.x - va.x) / dy, (vb.y - va.y) / dy, 1.0} : WorkVal{0.0, 0.0, 0.0};
      };
      const WorkVal wi_c = WI(ic, ie, uc, ue), wi_w = WI(iw, ic, uw, uc), wi_nw = WI(inw, in, unw, un),
                    wi_n = WI(in, ine, un, une);
      const WorkVal wj_c = WJ(ic, in, uc, un), wj_s = WJ(is, ic, us, uc), wj_se = WJ(ise, ie, use, ue),
                    wj_e = WJ(ie, ine, ue, une);
      // i-offset
      double Hf = (ic && ie) ? 0.5 * (Hc + He) : (ic ? Hc : He);
      if (Hf >= p.Hmin) {
        double u_x = wi_c.u, v_x = wi_c.v, u_y = 0.0, v_y = 0.0;
        double W = wj_c.w + wj_s.w + wj_se.w + wj_e.w;
        if (W > 0) {
          u_y = 1.0 / W * (wj_c.u + wj_s.u + wj_se.u + wj_e.u);
          v_y = 1.0 / W * (wj_c.v + wj_s.v + wj_se.v + wj_e.v);
        }
        double nu = 0.5 * B.x * pow(p.schoof_reg + second_invariant_2d(u_x, u_y, v_x, v_y), p.visc_power);
        r0 = nu * Hf;
      } else {
        r0 = p.notional;
      }
      // j-offset
      Hf = (ic && in) ? 0.5 * (Hc + Hn) : (ic ? Hc : Hn);
      if (Hf >= p.Hmin) {
        double u_y = wj_c.u, v_y = wj_c.v, u_x = 0.0, v_x = 0.0;
        double W = wi_c.w + wi_w.w + wi_nw.w + wi_n.w;
        if (W > 0.0) {
          u_x = 1.0 / W * (wi_c.u + wi_w.u + wi_nw.u + wi_n.u);
          v_x = 1.0 / W * (wi_c.v + wi_w.v + wi_nw.v + wi_n.v);
        }
        double nu = 0.5 * B.y * pow(p.schoof_reg + second_invariant_2d(u_x, u_y, v_x, v_y), p.visc_power);
        r1 = nu * Hf;
      } else {
        r1 = p.notional;
      }
      r0 *= p.enh_scaling;
      r0 += p.reg;
      r1 *= p.enh_scaling;
      r1 += p.reg;
    }
    const double2 old = nuH[k];
    if (p.underrelax != 1.0) {
      r0 *= p.underrelax;
      r0 += (1.0 - p.underrelax) * old.x;
      r1 *= p.underrelax;
      r1 += (1.0 - p.underrelax) * old.y;
    }
    nuH[k] = make_double2(r0, r1);
    if (p.with_norm) {
      const double wi = (i == 0 ? 1.0 : 0.0) + (i == g.Mx - 1 ? 1.0 : 0.0) + 1.0;
      const double wj = (j == 0 ? 1.0 : 0.0) + (j == g.My - 1 ? 1.0 : 0.0) + 1.0;
      const double w = wi * wj;
      acc[0] += fabs(r0) * w;
      acc[1] += fabs(r1) * w;
      acc[2] += fabs(old.x - r0) * w;
      acc[3] += fabs(old.y - r1) * w;
    }
    // basal drag for the next assembly (SSAFD.cc:744-759)
    const int Mc = mask[k];
    double bta = 0.0;
    if (m_grounded_ice(Mc))
      bta = basal_drag(c, tauc[k], uc.x, uc.y);
    else if (m_ice_free_land(Mc))
      bta = c.beta_ice_free_bedrock;
    if (c.sub_groundingline && m_icy(Mc)) bta = gl_mask[k] * basal_drag(c, tauc[k], uc.x, uc.y);
    beta[k] = bta;
  }
  if (p.with_norm) {
    double tot[4];
    if (grid_reduce<4>(acc, partials, ticket, tot)) {
      const double a = p.B_area;
      const double n0 = tot[0] * a, n1 = tot[1] * a, c0 = tot[2] * a, c1 = tot[3] * a;
      norm_out[0] = sqrt(n0 * n0 + n1 * n1);
      norm_out[1] = sqrt(c0 * c0 + c1 * c1);
    }
  }
}

// y = A x at cell (i, j) = tile position (ti, tj), x and nu*H staged in halo tiles
__device__ __forceinline__ double2 apply_cell_tile(const GridDev &g, const StencilConst &s, int i, int j, uint32_t f,
                                                   const HaloTile<double2> &xT, const HaloTile<double2> &nT,
                                                   double bta, int ti, int tj) {
  if (f & F_DIAG_ONLY) {
    const double2 xc = xT[ti + 1][tj + 1];
    return make_double2(s.scaling * xc.x, s.scaling * xc.y);
  }
  double c_w = nT[ti][tj + 1].x, c_e = nT[ti + 1][tj + 1].x, c_s = nT[ti + 1][tj].y, c_n = nT[ti + 1][tj + 1].y;
  if (f & F_NB_ANY) {   // nu_bedrock_set overrides (SSAFD.cc:561-585), from global memory
    const int k = cell(g, i, j);
    const double Hc = s.H[k], HE = s.H[nbr(g, i, j, 1, 0)];
    if (f & F_NB_W) c_w = s.nu_bedrock * 0.5 * (Hc + s.H[nbr(g, i, j, -1, 0)]);
    if (f & F_NB_E) c_e = s.nu_bedrock * 0.5 * (Hc + HE);
    if (f & F_NB_N) c_n = s.nu_bedrock * 0.5 * (Hc + s.H[nbr(g, i, j, 0, 1)]);
    if (f & F_NB_S) c_s = s.nu_bedrock * 0.5 * (Hc + HE);   // thickness(i+1, j), as SSAFD.cc:582
  }
  auto xr = [&](int di, int dj) { return xT[ti + 1 + di][tj + 1 + dj]; };
  if ((f & F_WEIGHTS) == F_WEIGHTS)
    return apply_regular<double, double2>(s.rdx2, s.rdy2, s.r2, s.r4, c_w, c_e, c_s, c_n, bta, xr);
  Row2 e1, e2;
  stencil_rows(s, f, c_w, c_e, c_s, c_n, bta, e1, e2);
  return apply_rows_rel<double, double2>(e1, e2, xr);
}

// Stage the x and nu*H halo tiles of tile t and load this thread's flags, beta and
// (optionally) one more vector entry `extra`, all in the same round trip to memory.
// Returns whether this thread's cell (i, j) lies inside the grid.
__device__ __forceinline__ bool stage_tile(const GridDev &g, const TileMap &tm, int t, const double2 *__restrict__ x,
                                           const double2 *__restrict__ nuH, const uint32_t *__restrict__ flags,
                                           const double *__restrict__ beta, const double2 *__restrict__ extra,
                                           HaloTile<double2> &xT, HaloTile<double2> &nT, int &i, int &j, int &k,
                                           uint32_t &f, double &bta, double2 &ex) {
  const int i0 = (t / tm.tiles_j) * TI, j0 = (t % tm.tiles_j) * TJ;
  i = i0 + (threadIdx.x >> 5);
  j = j0 + (threadIdx.x & 31);
  const bool inside = i < g.Mx && j < g.My;
  k = inside ? i * g.My + j : 0;
  f = flags[k];
  bta = beta[k];
  if (extra) ex = extra[k];
  __syncthreads();
  load_halo_tile<double2>(xT, i0, j0, g.Mx, g.My, [&](int a, int b) { return x[a * g.My + b]; });
  load_halo_tile<double2>(nT, i0, j0, g.Mx, g.My, [&](int a, int b) { return nuH[a * g.My + b]; });
  __syncthreads();
  return inside;
}

// y = A x (plain apply, for checking and for the residual of the refinement)
__global__ void __launch_bounds__(NT, 4) k_apply(GridDev g, TileMap tm, StencilConst s, const uint32_t *__restrict__ flags,
                                              const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                              const double2 *__restrict__ x, double2 *__restrict__ y) {
  __shared__ HaloTile<double2> xT, nT;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j, k;
    uint32_t f;
    double bta;
    double2 ex;
    if (!stage_tile(g, tm, t, x, nuH, flags, beta, nullptr, xT, nT, i, j, k, f, bta, ex)) continue;
    y[k] = apply_cell_tile(g, s, i, j, f, xT, nT, bta, threadIdx.x >> 5, threadIdx.x & 31);
  }
}

// block-diagonal (2x2) inverse for the point-block Jacobi preconditioner, and the
// zero-diagonal check of SSAFD.cc:766-776 (first offending cell index reported)
__global__ void __launch_bounds__(NT) k_diag_setup(GridDev g, TileMap tm, StencilConst s,
                                                   const uint32_t *__restrict__ flags,
                                                   const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                                   double4 *__restrict__ dinv, int *zero_diag_cell) {
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j;
    if (!tm.cell_of(g, t, i, j)) continue;
    const int k = cell(g, i, j);
    const uint32_t f = flags[k];
    if (f & F_DIAG_ONLY) {
      dinv[k] = make_double4(1.0 / s.scaling, 0.0, 0.0, 1.0 / s.scaling);
      continue;
    }
    double c_w, c_e, c_s, c_n;
    row_coefficients(g, s, i, j, f, nuH, c_w, c_e, c_s, c_n);
    Row2 e1, e2;
    stencil_rows(s, f, c_w, c_e, c_s, c_n, beta[k], e1, e2);
    const double a11 = e1.uC, a12 = e1.vC, a21 = e2.uC, a22 = e2.vC;
    if (fabs(a11) < 1e-16 || fabs(a22) < 1e-16) atomicMin(zero_diag_cell, k);
    const double det = a11 * a22 - a12 * a21;
    if (det != 0.0 && isfinite(det)) {
      const double r = 1.0 / det;
      dinv[k] = make_double4(a22 * r, -a12 * r, -a21 * r, a11 * r);
    } else {
      dinv[k] = make_double4(a11 != 0.0 ? 1.0 / a11 : 0.0, 0.0, 0.0, a22 != 0.0 ? 1.0 / a22 : 0.0);
    }
  }
}

// ---------------------------------------------------------------------------
// BiCGStab, right preconditioned by M^-1 = block-Jacobi (van der Vorst 1992),
// five kernels per iteration with all dot products fused into them.
// Stop: ||b - A x||_2 <= rtol ||b||_2 (the unpreconditioned norm of the
// reference's ASM path, SSAFD.cc:181-187).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT, 4) k_bicg_init(GridDev g, TileMap tm, StencilConst s,
                                                  const uint32_t *__restrict__ flags,
                                                  const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                                  const double2 *__restrict__ b, const double2 *__restrict__ x,
                                                  double2 *__restrict__ r, double2 *__restrict__ rhat,
                                                  double2 *__restrict__ p, double2 *__restrict__ v,
                                                  double *partials, unsigned *ticket, KState *st) {
  double acc[2] = {0.0, 0.0};
  __shared__ HaloTile<double2> xT, nT;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j, k;
    uint32_t f;
    double bta;
    double2 bk;
    if (!stage_tile(g, tm, t, x, nuH, flags, beta, b, xT, nT, i, j, k, f, bta, bk)) continue;
    const double2 ax = apply_cell_tile(g, s, i, j, f, xT, nT, bta, threadIdx.x >> 5, threadIdx.x & 31);
    const double2 rk = make_double2(bk.x - ax.x, bk.y - ax.y);
    r[k] = rk;
    rhat[k] = rk;
    p[k] = make_double2(0.0, 0.0);
    v[k] = make_double2(0.0, 0.0);
    acc[0] += dot2(rk, rk);
    acc[1] += dot2(bk, bk);
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    st->rnorm2 = tot[0];
    st->bnorm2 = tot[1];
    st->rnorm0 = sqrt(tot[0]);
    st->rho = tot[0];
    st->alpha = 1.0;
    st->omega = 1.0;
    st->beta = 0.0;
    st->iter = 0;
    st->status = 0;
    const double tol = st->rtol * sqrt(tot[1]);
    st->done = (sqrt(tot[0]) <= tol || tot[1] == 0.0) ? 1 : 0;
    if (!isfinite(tot[0])) { st->done = 1; st->status = KSP_NAN; }
  }
}

// p = r + beta (p - omega v);  phat = M^-1 p (block Jacobi; with multigrid phat is
// written by the V-cycle instead)
template <bool JAC>
__global__ void __launch_bounds__(NT) k_bicg_p(int N, const double2 *__restrict__ r, const double2 *__restrict__ v,
                                               const double4 *__restrict__ dinv, double2 *__restrict__ p,
                                               double2 *__restrict__ phat, const KState *st) {
  if (st->done) return;
  const double bta = st->beta, om = st->omega;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 rk = r[k], pk = p[k], vk = v[k];
    const double2 pn = make_double2(rk.x + bta * (pk.x - om * vk.x), rk.y + bta * (pk.y - om * vk.y));
    p[k] = pn;
    if (JAC) phat[k] = dmul(dinv[k], pn);
  }
}

// v = A phat; alpha = rho / (rhat . v)
__global__ void __launch_bounds__(NT, 4) k_bicg_v(GridDev g, TileMap tm, StencilConst s, const uint32_t *__restrict__ flags,
                                               const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                               const double2 *__restrict__ phat, const double2 *__restrict__ rhat,
                                               double2 *__restrict__ v, double *partials, unsigned *ticket,
                                               KState *st) {
  if (st->done) return;
  double acc[1] = {0.0};
  __shared__ HaloTile<double2> xT, nT;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j, k;
    uint32_t f;
    double bta;
    double2 ex;
    if (!stage_tile(g, tm, t, phat, nuH, flags, beta, nullptr, xT, nT, i, j, k, f, bta, ex)) continue;
    const double2 vk = apply_cell_tile(g, s, i, j, f, xT, nT, bta, threadIdx.x >> 5, threadIdx.x & 31);
    v[k] = vk;
    acc[0] += dot2(rhat[k], vk);
  }
  double tot[1];
  if (grid_reduce<1>(acc, partials, ticket, tot)) {
    if (tot[0] == 0.0 || !isfinite(tot[0])) {
      st->done = 1;
      st->status = isfinite(tot[0]) ? KSP_BREAKDOWN : KSP_NAN;
    } else {
      st->alpha = st->rho / tot[0];
    }
  }
}

// s = r - alpha v;  shat = M^-1 s
template <bool JAC>
__global__ void __launch_bounds__(NT) k_bicg_s(int N, const double2 *__restrict__ r, const double2 *__restrict__ v,
                                               const double4 *__restrict__ dinv, double2 *__restrict__ sv,
                                               double2 *__restrict__ shat, const KState *st) {
  if (st->done) return;
  const double al = st->alpha;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 rk = r[k], vk = v[k];
    const double2 sk = make_double2(rk.x - al * vk.x, rk.y - al * vk.y);
    sv[k] = sk;
    if (JAC) shat[k] = dmul(dinv[k], sk);
  }
}

// t = A shat; omega = (t . s) / (t . t)
__global__ void __launch_bounds__(NT, 4) k_bicg_t(GridDev g, TileMap tm, StencilConst s, const uint32_t *__restrict__ flags,
                                               const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                               const double2 *__restrict__ shat, const double2 *__restrict__ sv,
                                               double2 *__restrict__ tv, double *partials, unsigned *ticket,
                                               KState *st) {
  if (st->done) return;
  double acc[2] = {0.0, 0.0};
  __shared__ HaloTile<double2> xT, nT;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j, k;
    uint32_t f;
    double bta;
    double2 ex;
    if (!stage_tile(g, tm, t, shat, nuH, flags, beta, nullptr, xT, nT, i, j, k, f, bta, ex)) continue;
    const double2 tk = apply_cell_tile(g, s, i, j, f, xT, nT, bta, threadIdx.x >> 5, threadIdx.x & 31);
    tv[k] = tk;
    acc[0] += dot2(tk, sv[k]);
    acc[1] += dot2(tk, tk);
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) st->omega = (tot[1] != 0.0) ? tot[0] / tot[1] : 0.0;
}

// x += alpha phat + omega shat;  r = s - omega t;  convergence test
__global__ void __launch_bounds__(NT) k_bicg_x(int N, const double2 *__restrict__ phat, const double2 *__restrict__ shat,
                                               const double2 *__restrict__ sv, const double2 *__restrict__ tv,
                                               const double2 *__restrict__ rhat, double2 *__restrict__ x,
                                               double2 *__restrict__ r, double *partials, unsigned *ticket,
                                               KState *st) {
  if (st->done) return;
  const double al = st->alpha, om = st->omega;
  double acc[2] = {0.0, 0.0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 ph = phat[k], sh = shat[k], sk = sv[k], tk = tv[k];
    double2 xk = x[k];
    xk.x += al * ph.x + om * sh.x;
    xk.y += al * ph.y + om * sh.y;
    x[k] = xk;
    const double2 rk = make_double2(sk.x - om * tk.x, sk.y - om * tk.y);
    r[k] = rk;
    acc[0] += dot2(rhat[k], rk);
    acc[1] += dot2(rk, rk);
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    const double rho_new = tot[0];
    st->rnorm2 = tot[1];
    st->iter += 1;
    const double rn = sqrt(tot[1]), tol = st->rtol * sqrt(st->bnorm2);
    if (!isfinite(rn)) {
      st->done = 1; st->status = KSP_NAN;
    } else if (rn <= tol) {
      st->done = 1; st->status = 0;
    } else if (st->iter >= st->maxit) {
      st->done = 1; st->status = KSP_MAXIT;
    } else if (om == 0.0 || rho_new == 0.0) {
      st->done = 1; st->status = KSP_BREAKDOWN;
    } else {
      st->beta = (rho_new / st->rho) * (al / om);
      st->rho = rho_new;
    }
  }
}

// the outer residual of the mixed-precision refinement: r = b - A x in FP64, handed to the
// inner FP32 solve; the two norms feed the FP64 convergence test
__global__ void __launch_bounds__(NT, 4) k_residual32(GridDev g, TileMap tm, StencilConst s,
                                                      const uint32_t *__restrict__ flags,
                                                      const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                                      const double2 *__restrict__ b, const double2 *__restrict__ x,
                                                      float2 *__restrict__ r32, double *partials, unsigned *ticket,
                                                      double *out2) {
  double acc[2] = {0.0, 0.0};
  __shared__ HaloTile<double2> xT, nT;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j, k;
    uint32_t f;
    double bta;
    double2 bk;
    if (!stage_tile(g, tm, t, x, nuH, flags, beta, b, xT, nT, i, j, k, f, bta, bk)) continue;
    const double2 ax = apply_cell_tile(g, s, i, j, f, xT, nT, bta, threadIdx.x >> 5, threadIdx.x & 31);
    const double2 rk = make_double2(bk.x - ax.x, bk.y - ax.y);
    r32[k] = make_float2((float)rk.x, (float)rk.y);
    acc[0] += dot2(rk, rk);
    acc[1] += dot2(bk, bk);
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    out2[0] = tot[0];
    out2[1] = tot[1];
  }
}

__global__ void k_axpy32(int N, const float2 *__restrict__ d, double2 *__restrict__ x) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const float2 dk = d[k];
    double2 xk = x[k];
    xk.x += (double)dk.x;
    xk.y += (double)dk.y;
    x[k] = xk;
  }
}

// basal frictional heating (ShallowStressBalance.cc:179-205)
__global__ void k_bfrict(int N, pism_gpu_ssa_config c, const double2 *__restrict__ vel, const double *__restrict__ tauc,
                         const int8_t *__restrict__ mask, double *__restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    if (m_ocean(mask[k])) {
      out[k] = 0.0;
    } else {
      const double2 V = vel[k];
      const double C = basal_drag(c, tauc[k], V.x, V.y);
      const double bx = -C * V.x, by = -C * V.y;
      out[k] = -bx * V.x - by * V.y;
    }
  }
}

__global__ void k_scale(int n, double a, double *x) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) x[k] *= a;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int grid_for_tiles(const Launch &L, int tiles) { return tiles < L.max_blocks ? tiles : L.max_blocks; }
static int grid_for(const Launch &L, int n) {
  int b = (n + NT - 1) / NT;
  return b < L.max_blocks ? b : L.max_blocks;
}


void launch_convert_masks(const Launch &L, int N, const double *mask, const double *bc_mask, int8_t *mask_i,
                          uint8_t *bc_i) {
  L.tick();
  k_convert_masks<<<grid_for(L, N), NT, 0, L.stream>>>(N, mask, bc_mask, mask_i, bc_i);
}

void launch_prepare(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, int periodicity, const Fields &f) {
  L.tick();
  TileMap tm = make_tiles(g);
  k_prepare<<<grid_for_tiles(L, tm.tiles), NT, 0, L.stream>>>(g, tm, c, periodicity, f.H, f.srf, f.bed, f.mask,
                                                              f.bc, f.bcv, f.melange, f.taud, f.rhs, f.flags);
}

void launch_hardness(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const Fields &f, int Mz,
                     const double *z) {
  L.tick();
  int N = g.Mx * g.My;
  k_hardness<<<grid_for(L, N), NT, 0, L.stream>>>(g, N, c, f.H, f.mask, f.enthalpy, Mz, z, f.fracture, f.hardness);
}

void launch_nuH(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const Fields &f, double reg,
                double underrelax, bool with_norm, double *norm_out) {
  L.tick();
  TileMap tm = make_tiles(g);
  NuHParams p;
  const double n = c.ssa_Glen_exponent;
  p.reg = reg;
  p.underrelax = underrelax;
  p.Hmin = c.min_thickness_strength_extension_ssa;
  p.notional = c.constant_nu_strength_extension_ssa * c.min_thickness_strength_extension_ssa;
  p.schoof_reg = (c.Schoof_regularizing_velocity / c.Schoof_regularizing_length) *
                 (c.Schoof_regularizing_velocity / c.Schoof_regularizing_length);
  p.visc_power = (1.0 - n) / (2.0 * n);
  p.enh_scaling = 1.0 / pow(c.ssa_enhancement_factor, 1.0 / n);
  p.B_area = g.dx * g.dy;
  p.with_norm = with_norm ? 1 : 0;
  int blocks = grid_for_tiles(L, tm.tiles);
  if (c.calving_front_stress_boundary_condition)
    k_nuH<true><<<blocks, NT, 0, L.stream>>>(g, tm, c, p, f.vel, f.H, f.hardness, f.mask, f.tauc, f.gl_mask, f.nuH,
                                             f.beta, L.partials, L.ticket, norm_out);
  else
    k_nuH<false><<<blocks, NT, 0, L.stream>>>(g, tm, c, p, f.vel, f.H, f.hardness, f.mask, f.tauc, f.gl_mask, f.nuH,
                                              f.beta, L.partials, L.ticket, norm_out);
}

void launch_apply(const Launch &L, const GridDev &g, const Fields &f, const double2 *x, double2 *y) {
  L.tick();
  TileMap tm = make_tiles(g);
  k_apply<<<grid_for_tiles(L, tm.tiles), NT, 0, L.stream>>>(g, tm, stencil_const(g, f), f.flags, f.nuH, f.beta, x, y);
}

void launch_diag_setup(const Launch &L, const GridDev &g, const Fields &f, double4 *dinv, int *zero_diag_cell) {
  L.tick();
  TileMap tm = make_tiles(g);
  k_diag_setup<<<grid_for_tiles(L, tm.tiles), NT, 0, L.stream>>>(g, tm, stencil_const(g, f), f.flags, f.nuH, f.beta,
                                                                 dinv, zero_diag_cell);
}

void launch_bicg_init(const Launch &L, const GridDev &g, const Fields &f, const Krylov &K, const double2 *b,
                      const double2 *x) {
  L.tick();
  TileMap tm = make_tiles(g);
  k_bicg_init<<<grid_for_tiles(L, tm.tiles), NT, 0, L.stream>>>(g, tm, stencil_const(g, f), f.flags, f.nuH, f.beta, b,
                                                                x, K.r, K.rhat, K.p, K.v, L.partials, L.ticket, K.st);
}

void launch_bicg_iteration(const Launch &L, const GridDev &g, const Fields &f, const Krylov &K, double2 *x,
                           const MGHierarchy *mg, const LinePC *line) {
  L.tick(5);
  TileMap tm = make_tiles(g);
  const int N = g.Mx * g.My;
  const StencilConst s = stencil_const(g, f);
  const int bt = grid_for_tiles(L, tm.tiles), bv = grid_for(L, N);
  if (mg) {
    k_bicg_p<false><<<bv, NT, 0, L.stream>>>(N, K.r, K.v, K.dinv, K.p, K.phat, K.st);
    mg_vcycle(L, g, f, *mg, K.p, K.phat, K.st);
  } else if (line) {
    k_bicg_p<false><<<bv, NT, 0, L.stream>>>(N, K.r, K.v, K.dinv, K.p, K.phat, K.st);
    line_apply(L, g, *line, K.p, K.phat, K.st);
  } else {
    k_bicg_p<true><<<bv, NT, 0, L.stream>>>(N, K.r, K.v, K.dinv, K.p, K.phat, K.st);
  }
  k_bicg_v<<<bt, NT, 0, L.stream>>>(g, tm, s, f.flags, f.nuH, f.beta, K.phat, K.rhat, K.v, L.partials, L.ticket,
                                    K.st);
  if (mg) {
    k_bicg_s<false><<<bv, NT, 0, L.stream>>>(N, K.r, K.v, K.dinv, K.s, K.shat, K.st);
    mg_vcycle(L, g, f, *mg, K.s, K.shat, K.st);
  } else if (line) {
    k_bicg_s<false><<<bv, NT, 0, L.stream>>>(N, K.r, K.v, K.dinv, K.s, K.shat, K.st);
    line_apply(L, g, *line, K.s, K.shat, K.st);
  } else {
    k_bicg_s<true><<<bv, NT, 0, L.stream>>>(N, K.r, K.v, K.dinv, K.s, K.shat, K.st);
  }
  k_bicg_t<<<bt, NT, 0, L.stream>>>(g, tm, s, f.flags, f.nuH, f.beta, K.shat, K.s, K.t, L.partials, L.ticket, K.st);
  k_bicg_x<<<bv, NT, 0, L.stream>>>(N, K.phat, K.shat, K.s, K.t, K.rhat, x, K.r, L.partials, L.ticket, K.st);
}

void launch_residual32(const Launch &L, const GridDev &g, const Fields &f, const double2 *b, const double2 *x,
                       float2 *r32, double *out2) {
  L.tick();
  TileMap tm = make_tiles(g);
  k_residual32<<<grid_for_tiles(L, tm.tiles), NT, 0, L.stream>>>(g, tm, stencil_const(g, f), f.flags, f.nuH, f.beta, b,
                                                                 x, r32, L.partials, L.ticket, out2);
}

void launch_axpy32(const Launch &L, int N, const float2 *d, double2 *x) {
  L.tick();
  k_axpy32<<<grid_for(L, N), NT, 0, L.stream>>>(N, d, x);
}

void launch_bfrict(const Launch &L, int N, const pism_gpu_ssa_config &c, const Fields &f, double *out) {
  L.tick();
  k_bfrict<<<grid_for(L, N), NT, 0, L.stream>>>(N, c, f.vel, f.tauc, f.mask, out);
}

void launch_scale(const Launch &L, int n, double a, double *x) {
  L.tick();
  k_scale<<<grid_for(L, n), NT, 0, L.stream>>>(n, a, x);
}


// ---------------------------------------------------------------------------
// Restarted flexible GMRES(m) with right preconditioning (PETSc's KSPFGMRES; with a fixed
// preconditioner it is GMRES right-preconditioned, the reference's fallback set-up with
// the unpreconditioned residual norm, SSAFD.cc:164-219).  The Arnoldi basis is
// orthogonalised by classical Gram-Schmidt in one pass (PETSc's default, no refinement).
// The Givens rotations, the residual estimate |g[j+1]| and the tests run in the last
// block of the orthogonalisation kernel.  Stop: ||b - A x||_2 <= rtol ||b||_2.
// ---------------------------------------------------------------------------

// r = b - A x into V0.  init: the start of a solve (also ||b||); otherwise only after a
// cycle that ended without convergence (a restart).
__global__ void __launch_bounds__(NT, 4) k_gm_residual(GridDev g, TileMap tm, StencilConst s,
                                                    const uint32_t *__restrict__ flags,
                                                    const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                                    const double2 *__restrict__ b, const double2 *__restrict__ x,
                                                    double2 *__restrict__ v0, double *partials, unsigned *ticket,
                                                    KState *st, GState *gs, int init) {
  if (!init && (!gs->restart || st->done)) return;
  double acc[2] = {0.0, 0.0};
  __shared__ HaloTile<double2> xT, nT;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, j, k;
    uint32_t f;
    double bta;
    double2 bk;
    if (!stage_tile(g, tm, t, x, nuH, flags, beta, b, xT, nT, i, j, k, f, bta, bk)) continue;
    const double2 ax = apply_cell_tile(g, s, i, j, f, xT, nT, bta, threadIdx.x >> 5, threadIdx.x & 31);
    const double2 rk = make_double2(bk.x - ax.x, bk.y - ax.y);
    v0[k] = rk;
    acc[0] += dot2(rk, rk);
    acc[1] += dot2(bk, bk);
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    const double rn = sqrt(tot[0]);
    if (init) {
      gs->bnorm = sqrt(tot[1]);
      st->bnorm2 = tot[1];
      st->rnorm0 = rn;
      st->iter = 0;
      st->status = KSP_OK;
      st->done = 0;
    }
    st->rnorm2 = tot[0];
    gs->restart = 0;
    gs->need_update = 0;
    gs->cols = 0;
    for (int q = 0; q <= GM_MAXM; ++q) gs->g[q] = 0.0;
    gs->g[0] = rn;
    gs->scale0 = rn > 0.0 ? 1.0 / rn : 0.0;
    if (!isfinite(rn)) {
      st->done = 1;
      st->status = KSP_NAN;
      gs->scale0 = 0.0;
    } else if (rn <= st->rtol * gs->bnorm || gs->bnorm == 0.0) {
      st->done = 1;
      gs->scale0 = 0.0;
    }
  }
}

// V0 *= 1 / ||r0|| after a (re)start (scale0 is cleared by the next orthogonalisation)
__global__ void __launch_bounds__(NT) k_gm_scale0(int N, double2 *__restrict__ v0, const GState *gs) {
  const double sc = gs->scale0;
  if (sc == 0.0) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 v = v0[k];
    v0[k] = make_double2(v.x * sc, v.y * sc);
  }
}

// z = D^-1 v (point-block Jacobi)
__global__ void __launch_bounds__(NT) k_gm_jacobi(int N, const double2 *__restrict__ v,
                                                  const double4 *__restrict__ dinv, double2 *__restrict__ z,
                                                  const KState *st) {
  if (st && st->done) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) z[k] = dmul(dinv[k], v[k]);
}

// w = A z_j into V[j+1];  H[i][j] = <w, v_i> for i <= j
__global__ void __launch_bounds__(NT, 2) k_gm_apply_dots(GridDev g, TileMap tm, StencilConst s,
                                                      const uint32_t *__restrict__ flags,
                                                      const double2 *__restrict__ nuH,
                                                      const double *__restrict__ beta, const double2 *__restrict__ z,
                                                      const double2 *__restrict__ V, double2 *__restrict__ w, int j,
                                                      double *partials, unsigned *ticket, const KState *st,
                                                      GState *gs) {
  if (st->done) return;
  const size_t N = (size_t)g.Mx * g.My;
  double acc[GM_MAXM + 2];
#pragma unroll
  for (int q = 0; q < GM_MAXM + 2; ++q) acc[q] = 0.0;
  __shared__ HaloTile<double2> xT, nT;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int i, jj, k;
    uint32_t f;
    double bta;
    double2 ex;
    if (!stage_tile(g, tm, t, z, nuH, flags, beta, nullptr, xT, nT, i, jj, k, f, bta, ex)) continue;
    const double2 wk = apply_cell_tile(g, s, i, jj, f, xT, nT, bta, threadIdx.x >> 5, threadIdx.x & 31);
    w[k] = wk;
#pragma unroll
    for (int q = 0; q <= GM_MAXM; ++q)
      if (q <= j) acc[q] += dot2(V[q * N + k], wk);
  }
  double tot[GM_MAXM + 2];
  if (grid_reduce<GM_MAXM + 2>(acc, partials, ticket, tot))
    for (int q = 0; q <= j; ++q) gs->H[q][j] = tot[q];
}

// w -= sum_{i <= j} H[i][j] v_i;  h = ||w||;  rotations, residual estimate and tests
__global__ void __launch_bounds__(NT) k_gm_orth(int N, const double2 *__restrict__ V, double2 *__restrict__ w, int j,
                                                int m, double *partials, unsigned *ticket, KState *st, GState *gs) {
  if (st->done) return;
  __shared__ double hcol[GM_MAXM + 1];
  if (threadIdx.x <= j) hcol[threadIdx.x] = gs->H[threadIdx.x][j];
  __syncthreads();
  double acc[1] = {0.0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    double2 wk = w[k];
#pragma unroll
    for (int q = 0; q <= GM_MAXM; ++q)
      if (q <= j) {
        const double2 v = V[(size_t)q * N + k];
        wk.x -= hcol[q] * v.x;
        wk.y -= hcol[q] * v.y;
      }
    w[k] = wk;
    acc[0] += dot2(wk, wk);
  }
  double tot[1];
  if (!grid_reduce<1>(acc, partials, ticket, tot)) return;
  const double hn = sqrt(tot[0]);
  gs->hnext = hn;
  gs->scale0 = 0.0;
  for (int i = 0; i < j; ++i) {
    const double a = gs->H[i][j], b = gs->H[i + 1][j];
    gs->H[i][j] = gs->cs[i] * a + gs->sn[i] * b;
    gs->H[i + 1][j] = -gs->sn[i] * a + gs->cs[i] * b;
  }
  const double a = gs->H[j][j], r = hypot(a, hn);
  st->iter += 1;
  if (!isfinite(hn) || !isfinite(r)) {
    st->done = 1;
    st->status = KSP_NAN;
    gs->need_update = 0;
    return;
  }
  if (r == 0.0) {   // the new direction and its projection both vanish: nothing to add
    st->done = 1;
    st->status = KSP_BREAKDOWN;
    gs->cols = j;
    gs->need_update = j > 0;
    return;
  }
  const double c = a / r, sg = hn / r;
  gs->cs[j] = c;
  gs->sn[j] = sg;
  gs->H[j][j] = r;
  gs->H[j + 1][j] = 0.0;
  const double gj = gs->g[j];
  gs->g[j] = c * gj;
  gs->g[j + 1] = -sg * gj;
  const double res = fabs(gs->g[j + 1]);
  st->rnorm2 = res * res;
  gs->cols = j + 1;
  if (res <= st->rtol * gs->bnorm || hn == 0.0) {
    st->done = 1;
    st->status = KSP_OK;
    gs->need_update = 1;
  } else if (st->iter >= st->maxit) {
    st->done = 1;
    st->status = KSP_MAXIT;
    gs->need_update = 1;
  } else if (j + 1 == m) {
    gs->restart = 1;
    gs->need_update = 1;
  }
}

// V[j+1] *= 1 / h_{j+1,j} while the cycle goes on
__global__ void __launch_bounds__(NT) k_gm_scale_next(int N, double2 *__restrict__ w, const KState *st,
                                                      const GState *gs) {
  if (st->done || gs->restart) return;
  const double sc = 1.0 / gs->hnext;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 v = w[k];
    w[k] = make_double2(v.x * sc, v.y * sc);
  }
}

// R y = g over the finished columns (one thread; at most 30 x 30)
__global__ void k_gm_solve(GState *gs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (!gs->need_update) {
    gs->cols_upd = 0;
    return;
  }
  const int n = gs->cols;
  for (int i = n - 1; i >= 0; --i) {
    double a = gs->g[i];
    for (int q = i + 1; q < n; ++q) a -= gs->H[i][q] * gs->y[q];
    gs->y[i] = a / gs->H[i][i];
  }
  gs->cols_upd = n;
  gs->need_update = 0;
}

// x += sum_{i < cols} y_i z_i
__global__ void __launch_bounds__(NT) k_gm_update(int N, const double2 *__restrict__ Z, double2 *__restrict__ x,
                                                  const GState *gs) {
  const int n = gs->cols_upd;
  if (n == 0) return;
  __shared__ double ys[GM_MAXM];
  if (threadIdx.x < n) ys[threadIdx.x] = gs->y[threadIdx.x];
  __syncthreads();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    double2 xk = x[k];
#pragma unroll
    for (int q = 0; q < GM_MAXM; ++q)
      if (q < n) {
        const double2 zv = Z[(size_t)q * N + k];
        xk.x += ys[q] * zv.x;
        xk.y += ys[q] * zv.y;
      }
    x[k] = xk;
  }
}

void launch_gmres_residual(const Launch &L, const GridDev &g, const Fields &f, const Gmres &G, const double2 *b,
                           const double2 *x, int init) {
  L.tick(2);
  TileMap tm = make_tiles(g);
  const int N = g.Mx * g.My;
  k_gm_residual<<<grid_for_tiles(L, tm.tiles), NT, 0, L.stream>>>(g, tm, stencil_const(g, f), f.flags, f.nuH, f.beta,
                                                                  b, x, G.V, G.partials, L.ticket, G.st, G.gs, init);
  k_gm_scale0<<<grid_for(L, N), NT, 0, L.stream>>>(N, G.V, G.gs);
}

void launch_gmres_precondition(const Launch &L, const GridDev &g, const Fields &f, const Gmres &G,
                               const double4 *dinv, const MGHierarchy *mg, const LinePC *line, int j) {
  const int N = g.Mx * g.My;
  const double2 *vj = G.V + (size_t)j * N;
  double2 *zj = G.Z + (size_t)j * N;
  if (mg) {
    mg_vcycle(L, g, f, *mg, vj, zj, G.st);
  } else if (line) {
    line_apply(L, g, *line, vj, zj, G.st);
  } else {
    L.tick();
    k_gm_jacobi<<<grid_for(L, N), NT, 0, L.stream>>>(N, vj, dinv, zj, G.st);
  }
}

void launch_gmres_orthogonalize(const Launch &L, const GridDev &g, const Fields &f, const Gmres &G, int j) {
  L.tick(3);
  TileMap tm = make_tiles(g);
  const int N = g.Mx * g.My;
  double2 *zj = G.Z + (size_t)j * N, *w = G.V + (size_t)(j + 1) * N;
  k_gm_apply_dots<<<grid_for_tiles(L, tm.tiles), NT, 0, L.stream>>>(g, tm, stencil_const(g, f), f.flags, f.nuH, f.beta,
                                                                    zj, G.V, w, j, G.partials, L.ticket, G.st, G.gs);
  k_gm_orth<<<grid_for(L, N), NT, 0, L.stream>>>(N, G.V, w, j, G.m, G.partials, L.ticket, G.st, G.gs);
  k_gm_scale_next<<<grid_for(L, N), NT, 0, L.stream>>>(N, w, G.st, G.gs);
}

void launch_gmres_step(const Launch &L, const GridDev &g, const Fields &f, const Gmres &G, const double4 *dinv,
                       const MGHierarchy *mg, const LinePC *line, int j) {
  launch_gmres_precondition(L, g, f, G, dinv, mg, line, j);
  launch_gmres_orthogonalize(L, g, f, G, j);
}

// r = v - y where y = A z (the residual the learned correction sees); skipped once done
__global__ void k_pc_residual(int N, const double2 *__restrict__ v, double2 *__restrict__ y, const KState *st) {
  if (st && st->done) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 vk = v[k], yk = y[k];
    y[k] = make_double2(vk.x - yk.x, vk.y - yk.y);
  }
}

// gamma = (r, Ad) / (Ad, Ad) (0 when Ad vanishes), the step along d that minimises
// ||r - gamma A d||; then z += gamma d
__global__ void k_pc_gamma(int N, const double2 *__restrict__ r, const double2 *__restrict__ ad, double *partials,
                           unsigned *ticket, double *gamma, const KState *st) {
  if (st && st->done) return;
  double acc[2] = {0.0, 0.0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 rk = r[k], a = ad[k];
    acc[0] += rk.x * a.x + rk.y * a.y;
    acc[1] += a.x * a.x + a.y * a.y;
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) *gamma = (tot[1] > 0.0 && isfinite(tot[0] / tot[1])) ? tot[0] / tot[1] : 0.0;
}

__global__ void k_pc_add(int N, const double2 *__restrict__ d, const double *__restrict__ gamma,
                         double2 *__restrict__ z, const KState *st) {
  if (st && st->done) return;
  const double gm = *gamma;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 dk = d[k], zk = z[k];
    z[k] = make_double2(zk.x + gm * dk.x, zk.y + gm * dk.y);
  }
}

void launch_pc_line_search(const Launch &L, const GridDev &g, const Fields &f, const double2 *r, const double2 *d,
                           double2 *ad, double *gamma, double2 *z, const KState *st) {
  launch_apply(L, g, f, d, ad);
  L.tick(2);
  const int N = g.Mx * g.My;
  k_pc_gamma<<<grid_for(L, N), NT, 0, L.stream>>>(N, r, ad, L.partials, L.ticket, gamma, st);
  k_pc_add<<<grid_for(L, N), NT, 0, L.stream>>>(N, d, gamma, z, st);
}

void launch_pc_residual(const Launch &L, const GridDev &g, const Fields &f, const double2 *v, const double2 *z,
                        double2 *r, const KState *st) {
  launch_apply(L, g, f, z, r);
  L.tick();
  const int N = g.Mx * g.My;
  k_pc_residual<<<grid_for(L, N), NT, 0, L.stream>>>(N, v, r, st);
}

void launch_pc_apply(const Launch &L, const GridDev &g, const Fields &f, const double4 *dinv, const MGHierarchy *mg,
                     const LinePC *line, const double2 *r, double2 *z) {
  const int N = g.Mx * g.My;
  if (mg) {
    mg_vcycle(L, g, f, *mg, r, z, nullptr);
  } else if (line) {
    line_apply(L, g, *line, r, z, nullptr);
  } else {
    L.tick();
    k_gm_jacobi<<<grid_for(L, N), NT, 0, L.stream>>>(N, r, dinv, z, nullptr);
  }
}

void launch_gmres_update(const Launch &L, const GridDev &g, const Gmres &G, double2 *x) {
  L.tick(2);
  const int N = g.Mx * g.My;
  k_gm_solve<<<1, 32, 0, L.stream>>>(G.gs);
  k_gm_update<<<grid_for(L, N), NT, 0, L.stream>>>(N, G.Z, x, G.gs);
}

// sets the WHILE condition of a graph-resident Krylov loop from the device state
__global__ void k_loop_condition(cudaGraphConditionalHandle cond, const KState *st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) cudaGraphSetConditional(cond, st->done ? 0u : 1u);
}

void launch_loop_condition(const Launch &L, cudaGraphConditionalHandle cond, const KState *st) {
  L.tick();
  k_loop_condition<<<1, 32, 0, L.stream>>>(cond, st);
}

}  // namespace pism_gpu
