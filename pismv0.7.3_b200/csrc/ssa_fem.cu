// ssa_fem.cu — the Q1 finite-element SSA (SSAFEM.cc:151-840, FETools.cc/.hh) on the GPU:
// the coefficients cached at the 2 x 2 Gauss points of each element
// (SSAFEM::cacheQuadPtValues, SSAFEM.cc:233-375), the weak-form residual
// (compute_local_function, :441-532) and its Newton Jacobian (compute_local_jacobian,
// :571-700), Dirichlet rows scale (u - u_bc) with their columns dropped (DirichletData_Vector,
// FETools.cc:671-741), and the linear solves of the Newton steps by conjugate gradients with
// the inverse 2 x 2 diagonal blocks as preconditioner.
//
// Layout: the residual and Jacobian are assembled per node, not per element.  One thread owns
// node (i, j) and walks the (up to) four elements around it in the reference's element order
// ((i-1, j-1), (i-1, j), (i, j-1), (i, j): i outer), computing each element's quadrature
// values and adding the element's row block for this node, so the sums are deterministic and
// no element buffer or atomic is needed; the price is each element's quadrature evaluated by
// its four nodes.  The Jacobian is stored as 9 neighbour blocks of 2 x 2 per node,
// structure-of-arrays ([36][N]), which the CG apply reads coalesced.
#include <algorithm>

#include "ssa_fem.h"
#include "ssa_reduce.cuh"

namespace pism_gpu {

namespace {

constexpr int NTF = RED_THREADS;

// the element-local node offsets of DOFMap (FETools.cc:206-207)
__constant__ int kDI[4] = {0, 1, 1, 0};
__constant__ int kDJ[4] = {0, 0, 1, 1};

struct FemGrid {
  int Mx, My, nex, ney, px, py;   // px, py: periodic in x / y
};

__device__ __forceinline__ int fem_node(const FemGrid &G, int i, int j) {
  return wrap(i, G.Mx) * G.My + wrap(j, G.My);
}

// FlowLaw::averaged_hardness (flowlaws.cc:141-185) over the enthalpy column interpolated to a
// quadrature point from the element's four node columns, Enth_q[k] = sum_p val[p] E_p[k]
// (SSAFEM.cc:326-339)
__device__ double fem_averaged_hardness(const pism_gpu_ssa_config &c, double H, const double *z, int Mz,
                                        const double *E[4], const double val[4]) {
  int kb = 0, hi = Mz - 1;   // kBelowHeight: largest k in [0, Mz-2] with z[k] <= H
  while (hi > kb + 1) {
    const int mid = (kb + hi) / 2;
    if (z[mid] > H) hi = mid; else kb = mid;
  }
  auto Eq = [&](int k) {
    double e = 0.0;
    for (int p = 0; p < 4; ++p) e += val[p] * E[p][k];
    return e;
  };
  double B = 0.0;
  if (kb > 0) {
    double h0 = hardness_parameter(c, Eq(0), ec_pressure(c, H));
    for (int k = 1; k <= kb; ++k) {
      const double h1 = hardness_parameter(c, Eq(k), ec_pressure(c, H - z[k]));
      B += (z[k] - z[k - 1]) * (h0 + h1);
      h0 = h1;
    }
  }
  B *= 0.5;
  const double depth = H - z[kb];
  B += depth * hardness_parameter(c, Eq(kb), ec_pressure(c, depth));
  return H > 0 ? B / H : 0.0;
}

// SSAFEM::cacheQuadPtValues (SSAFEM.cc:233-375): one thread per element
__global__ void __launch_bounds__(NTF) k_fem_coefficients(FemGrid G, pism_gpu_ssa_config c, FemGerms W,
                                                          FemCoef C, const double *H, const double *bed,
                                                          const double *tauc, const double *srf,
                                                          const double *enthalpy, const double *z, int Mz,
                                                          double icefree_thickness, double is_floating_thickness) {
  const int Ne = G.nex * G.ney;
  const double alpha = 1.0 - c.ice_density / c.sea_water_density;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Ne; e += gridDim.x * blockDim.x) {
    const int ei = e / G.ney, ej = e - ei * G.ney;
    int n[4];
    for (int k = 0; k < 4; ++k) n[k] = fem_node(G, ei + kDI[k], ej + kDJ[k]);
    for (int q = 0; q < 4; ++q) {
      double Hq = 0, bq = 0, tq = 0, hx = 0, hy = 0;
      for (int k = 0; k < 4; ++k) {   // Quadrature_Scalar::computeTrialFunctionValues
        Hq += W.val[q][k] * H[n[k]];
        bq += W.val[q][k] * bed[n[k]];
        tq += W.val[q][k] * tauc[n[k]];
        hx += W.gx[q][k] * srf[n[k]];
        hy += W.gy[q][k] * srf[n[k]];
      }
      const int o = q * Ne + e;
      C.H[o] = Hq;
      C.tauc[o] = tq;
      C.tdu[o] = -c.ice_density * c.standard_gravity * Hq * hx;
      C.tdv[o] = -c.ice_density * c.standard_gravity * Hq * hy;
      // GeometryCalculator::mask (Mask.hh:82-118), dry simulation off
      const double hgrounded = bq + Hq, hfloating = c.sea_level + alpha * Hq;
      const bool floating = hfloating > hgrounded + is_floating_thickness, ice_free = Hq < icefree_thickness;
      C.mask[o] = (int8_t)(floating ? (ice_free ? MASK_ICE_FREE_OCEAN : MASK_FLOATING)
                                    : (ice_free ? MASK_ICE_FREE_BEDROCK : MASK_GROUNDED));
      if (c.flow_law == PISM_FLOW_LAW_ISOTHERMAL_GLEN) {
        C.B[o] = pow(c.ice_softness, -1.0 / c.ssa_Glen_exponent);
      } else {
        const double *E[4] = {enthalpy + (size_t)n[0] * Mz, enthalpy + (size_t)n[1] * Mz,
                              enthalpy + (size_t)n[2] * Mz, enthalpy + (size_t)n[3] * Mz};
        C.B[o] = fem_averaged_hardness(c, Hq, z, Mz, E, W.val[q]);
      }
    }
  }
}

// SSAFEM::PointwiseNuHAndBeta (SSAFEM.cc:393-432) with FlowLaw::effective_viscosity
// (flowlaws.hh:100-112) and drag_with_derivative (basal_resistance.cc:59-68, 174-190)
struct Pointwise {
  double eta, deta, beta, dbeta;
};

__device__ __forceinline__ Pointwise nuH_and_beta(const FemProblem &P, double H, double B, double tauc, int mask,
                                                  double u, double v, const double Du[3]) {
  const pism_gpu_ssa_config &c = P.c;
  Pointwise w;
  if (H < c.min_thickness_strength_extension_ssa) {
    w.eta = P.notional_strength;
    w.deta = 0.0;
  } else {
    const double n = c.ssa_Glen_exponent, power = (1.0 - n) / (2.0 * n);
    const double reg = (c.Schoof_regularizing_velocity / c.Schoof_regularizing_length) *
                       (c.Schoof_regularizing_velocity / c.Schoof_regularizing_length);
    // secondInvariantDu_2D, flowlaws.hh:42-44
    const double gamma = 0.5 * (Du[0] * Du[0] + Du[1] * Du[1] + (Du[0] + Du[1]) * (Du[0] + Du[1]) +
                                2 * Du[2] * Du[2]);
    const double nu = 0.5 * B * pow(reg + gamma, power);
    w.eta = c.epsilon_ssa + nu * H;
    w.deta = power * nu / (reg + gamma) * H;
  }
  if (m_grounded_ice(mask)) {
    const double magreg2 = c.plastic_regularization * c.plastic_regularization + u * u + v * v;
    if (!c.do_pseudo_plastic_till) {
      w.beta = tauc / sqrt(magreg2);
      w.dbeta = -1 * w.beta / magreg2;
    } else {
      const double q = c.pseudo_plastic_q;
      if (c.sliding_scale_factor_reduces_tauc > 0.0) {
        const double Aq = pow(c.sliding_scale_factor_reduces_tauc, q);
        w.beta = (tauc / Aq) * pow(magreg2, 0.5 * (q - 1)) * pow(c.pseudo_plastic_uthreshold, -q);
      } else {
        w.beta = tauc * pow(magreg2, 0.5 * (q - 1)) * pow(c.pseudo_plastic_uthreshold, -q);
      }
      w.dbeta = (q - 1) * w.beta / magreg2;
    }
  } else {
    w.beta = m_ice_free_land(mask) ? c.beta_ice_free_bedrock : 0.0;
    w.dbeta = 0.0;
  }
  return w;
}

// The residual (compute_local_function, SSAFEM.cc:441-532) and, with JAC, the Jacobian rows
// (compute_local_jacobian, :571-700) of one node, summed over its elements in the reference's
// element order; ||F||^2 over the grid in block order.
template <bool JAC>
__global__ void __launch_bounds__(NTF) k_fem_node(FemProblem P, FemGrid G, FemCoef C, const double2 *vel,
                                                  const uint8_t *bc, const double2 *bcv, double2 *F, double *J,
                                                  double4 *dinv, int *zero_pivot, FemScalars *sc,
                                                  double *partials, unsigned *ticket) {
  const int N = G.Mx * G.My, Ne = G.nex * G.ney;
  const FemGerms &W = P.W;
  double acc[1] = {0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const int i = n / G.My, j = n - i * G.My;
    double Jn[9][2][2];
    if (JAC)
      for (int b = 0; b < 9; ++b) Jn[b][0][0] = Jn[b][0][1] = Jn[b][1][0] = Jn[b][1][1] = 0.0;
    double2 Fn = make_double2(0.0, 0.0);
    if (bc[n]) {   // DirichletData_Vector::fix_residual / fix_jacobian (FETools.cc:702-741)
      const double2 x = vel[n], b = bcv[n];
      Fn = make_double2(P.scale * (x.x - b.x), P.scale * (x.y - b.y));
      if (JAC) Jn[4][0][0] = Jn[4][1][1] = P.scale;
    } else {
      // the elements around the node, in element order; k: the node's place in each
      const int erel[4][2] = {{-1, -1}, {-1, 0}, {0, -1}, {0, 0}};
      const int kloc[4] = {2, 1, 3, 0};
      for (int t = 0; t < 4; ++t) {
        int ei = i + erel[t][0], ej = j + erel[t][1];
        if (G.px) ei = wrap(ei, G.Mx); else if (ei < 0 || ei >= G.nex) continue;
        if (G.py) ej = wrap(ej, G.My); else if (ej < 0 || ej >= G.ney) continue;
        const int e = ei * G.ney + ej, k = kloc[t];
        double2 xl[4];
        bool lbc[4];
        for (int l = 0; l < 4; ++l) {   // DirichletData_Vector::update (FETools.cc:680-692)
          const int nl = fem_node(G, ei + kDI[l], ej + kDJ[l]);
          lbc[l] = bc[nl] != 0;
          xl[l] = lbc[l] ? bcv[nl] : vel[nl];
        }
        double ru = 0.0, rv = 0.0;
        double K[2][4][2];
        if (JAC)
          for (int l = 0; l < 4; ++l) K[0][l][0] = K[0][l][1] = K[1][l][0] = K[1][l][1] = 0.0;
        for (int q = 0; q < 4; ++q) {
          // Quadrature_Vector::computeTrialFunctionValues (FETools.cc:431-446)
          double u = 0, v = 0, Du[3] = {0, 0, 0};
          for (int l = 0; l < 4; ++l) {
            u += W.val[q][l] * xl[l].x;
            v += W.val[q][l] * xl[l].y;
            Du[0] += W.gx[q][l] * xl[l].x;
            Du[1] += W.gy[q][l] * xl[l].y;
            Du[2] += 0.5 * (W.gy[q][l] * xl[l].x + W.gx[q][l] * xl[l].y);
          }
          const int o = q * Ne + e;
          const Pointwise pw = nuH_and_beta(P, C.H[o], C.B[o], C.tauc[o], C.mask[o], u, v, Du);
          const double jw = W.JxW[q];
          const double Ux = Du[0], Vy = Du[1], UyVx = 2.0 * Du[2];
          const double psi = W.val[q][k], psx = W.gx[q][k], psy = W.gy[q][k];
          const double tbu = u * (-pw.beta), tbv = v * (-pw.beta);
          ru += jw * (pw.eta * (psx * (4.0 * Ux + 2.0 * Vy) + psy * UyVx) - psi * (tbu + C.tdu[o]));
          rv += jw * (pw.eta * (psx * UyVx + psy * (2.0 * Ux + 4.0 * Vy)) - psi * (tbv + C.tdv[o]));
          if (JAC) {
            for (int l = 0; l < 4; ++l) {
              const double phi = W.val[q][l], phx = W.gx[q][l], phy = W.gy[q][l];
              const double gamma_u = (2.0 * Ux + Vy) * phx + Du[2] * phy;
              const double gamma_v = Du[2] * phx + (Ux + 2.0 * Vy) * phy;
              const double eta_u = pw.deta * gamma_u, eta_v = pw.deta * gamma_v;
              const double taub_xu = -pw.dbeta * u * u * phi - pw.beta * phi;
              const double taub_xv = -pw.dbeta * u * v * phi;
              const double taub_yu = -pw.dbeta * v * u * phi;
              const double taub_yv = -pw.dbeta * v * v * phi - pw.beta * phi;
              K[0][l][0] += jw * (eta_u * (psx * (4 * Ux + 2 * Vy) + psy * UyVx) +
                                  pw.eta * (4 * psx * phx + psy * phy) - psi * taub_xu);
              K[0][l][1] += jw * (eta_v * (psx * (4 * Ux + 2 * Vy) + psy * UyVx) +
                                  pw.eta * (2 * psx * phy + psy * phx) - psi * taub_xv);
              K[1][l][0] += jw * (eta_u * (psx * UyVx + psy * (2 * Ux + 4 * Vy)) +
                                  pw.eta * (psx * phy + 2 * psy * phx) - psi * taub_yu);
              K[1][l][1] += jw * (eta_v * (psx * UyVx + psy * (2 * Ux + 4 * Vy)) +
                                  pw.eta * (psx * phx + 4 * psy * phy) - psi * taub_yv);
            }
          }
        }
        Fn.x += ru;   // DOFMap::addLocalResidualBlock
        Fn.y += rv;
        if (JAC)
          for (int l = 0; l < 4; ++l) {
            if (lbc[l]) continue;   // Dirichlet columns are left out (DirichletData::constrain)
            const int b = (erel[t][0] + kDI[l] + 1) * 3 + (erel[t][1] + kDJ[l] + 1);
            Jn[b][0][0] += K[0][l][0];
            Jn[b][0][1] += K[0][l][1];
            Jn[b][1][0] += K[1][l][0];
            Jn[b][1][1] += K[1][l][1];
          }
      }
    }
    F[n] = Fn;
    acc[0] += Fn.x * Fn.x + Fn.y * Fn.y;
    if (JAC) {
      for (int b = 0; b < 9; ++b)
        for (int r = 0; r < 2; ++r)
          for (int s = 0; s < 2; ++s) J[(size_t)(b * 4 + r * 2 + s) * N + n] = Jn[b][r][s];
      const double a = Jn[4][0][0], b = Jn[4][0][1], cc = Jn[4][1][0], d = Jn[4][1][1];
      const double det = a * d - b * cc;
      if (det == 0.0 || !isfinite(det)) {
        *zero_pivot = n + 1;
        dinv[n] = make_double4(0.0, 0.0, 0.0, 0.0);
      } else {
        dinv[n] = make_double4(d / det, -b / det, -cc / det, a / det);
      }
    }
  }
  double tot[1];
  if (grid_reduce<1>(acc, partials, ticket, tot)) sc->f2 = tot[0];
}

// ---- conjugate gradients on J du = -F, preconditioned by the inverse diagonal blocks ----
__device__ __forceinline__ double2 bmul(double4 A, double2 x) {
  return make_double2(A.x * x.x + A.y * x.y, A.z * x.x + A.w * x.y);
}

__global__ void __launch_bounds__(NTF) k_cg_init(int N, const double2 *F, const double4 *dinv, double2 *x,
                                                 double2 *r, double2 *z, double2 *p, FemCG *cg, double rtol,
                                                 int maxit, double *partials, unsigned *ticket) {
  double acc[2] = {0.0, 0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const double2 rn = make_double2(-F[n].x, -F[n].y), zn = bmul(dinv[n], rn);
    x[n] = make_double2(0.0, 0.0);
    r[n] = rn;
    z[n] = zn;
    p[n] = zn;
    acc[0] += rn.x * zn.x + rn.y * zn.y;
    acc[1] += rn.x * rn.x + rn.y * rn.y;
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    cg->rz = tot[0];
    cg->bb = tot[1];
    cg->rr = tot[1];
    cg->rtol = rtol;
    cg->maxit = maxit;
    cg->its = 0;
    cg->done = tot[1] == 0.0 ? 1 : 0;
  }
}

__global__ void __launch_bounds__(NTF) k_cg_apply(FemGrid G, const double *J, const double2 *p, double2 *q,
                                                  FemCG *cg, double *partials, unsigned *ticket) {
  if (cg->done) return;   // uniform over the grid: set by an earlier kernel
  const int N = G.Mx * G.My;
  double acc[1] = {0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const int i = n / G.My, j = n - i * G.My;
    double2 y = make_double2(0.0, 0.0);
    for (int b = 0; b < 9; ++b) {
      const double2 x = p[fem_node(G, i + b / 3 - 1, j + b % 3 - 1)];
      y.x += J[(size_t)(b * 4 + 0) * N + n] * x.x + J[(size_t)(b * 4 + 1) * N + n] * x.y;
      y.y += J[(size_t)(b * 4 + 2) * N + n] * x.x + J[(size_t)(b * 4 + 3) * N + n] * x.y;
    }
    q[n] = y;
    const double2 pn = p[n];
    acc[0] += pn.x * y.x + pn.y * y.y;
  }
  double tot[1];
  if (grid_reduce<1>(acc, partials, ticket, tot)) {
    cg->pq = tot[0];
    if (!(tot[0] > 0.0)) cg->done = 2;   // J not positive definite along p
    else cg->alpha = cg->rz / tot[0];
  }
}

__global__ void __launch_bounds__(NTF) k_cg_update(int N, const double4 *dinv, const double2 *p, const double2 *q,
                                                   double2 *x, double2 *r, double2 *z, FemCG *cg, double *partials,
                                                   unsigned *ticket) {
  if (cg->done) return;
  const double alpha = cg->alpha;
  double acc[2] = {0.0, 0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const double2 pn = p[n], qn = q[n];
    double2 xn = x[n], rn = r[n];
    xn.x += alpha * pn.x;
    xn.y += alpha * pn.y;
    rn.x -= alpha * qn.x;
    rn.y -= alpha * qn.y;
    const double2 zn = bmul(dinv[n], rn);
    x[n] = xn;
    r[n] = rn;
    z[n] = zn;
    acc[0] += rn.x * zn.x + rn.y * zn.y;
    acc[1] += rn.x * rn.x + rn.y * rn.y;
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    cg->beta = tot[0] / cg->rz;
    cg->rz = tot[0];
    cg->rr = tot[1];
    cg->its += 1;
    if (tot[1] <= cg->rtol * cg->rtol * cg->bb) cg->done = 1;
    else if (cg->its >= cg->maxit) cg->done = 3;
  }
}

__global__ void __launch_bounds__(NTF) k_cg_direction(int N, const double2 *z, double2 *p, const FemCG *cg) {
  if (cg->done) return;
  const double beta = cg->beta;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const double2 zn = z[n], pn = p[n];
    p[n] = make_double2(zn.x + beta * pn.x, zn.y + beta * pn.y);
  }
}

// trial = vel + lambda du, with ||lambda du||^2 and ||trial||^2
__global__ void __launch_bounds__(NTF) k_fem_trial(int N, const double2 *vel, const double2 *du, double lambda,
                                                   double2 *trial, FemScalars *sc, double *partials,
                                                   unsigned *ticket) {
  double acc[2] = {0.0, 0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const double2 s = make_double2(lambda * du[n].x, lambda * du[n].y), v = vel[n];
    const double2 t = make_double2(v.x + s.x, v.y + s.y);
    trial[n] = t;
    acc[0] += s.x * s.x + s.y * s.y;
    acc[1] += t.x * t.x + t.y * t.y;
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    sc->step2 = tot[0];
    sc->x2 = tot[1];
  }
}

FemGrid fem_grid(const FemProblem &P) {
  FemGrid G;
  G.Mx = P.Mx;
  G.My = P.My;
  G.px = (P.periodicity & 1) ? 1 : 0;
  G.py = (P.periodicity & 2) ? 1 : 0;
  G.nex = G.px ? P.Mx : P.Mx - 1;   // ElementMap, FETools.cc:38-83
  G.ney = G.py ? P.My : P.My - 1;
  return G;
}

int blocks(const Launch &L, int n) { return std::max(1, std::min((n + NTF - 1) / NTF, L.max_blocks)); }

template <typename T>
int alloc(T **p, size_t count) {
  return cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1)) == cudaSuccess ? 0 : 1;
}

}  // namespace

FemGerms fem_germs(double dx, double dy) {
  // ShapeQ1 (FETools.hh:187-213) at the Gauss points (FETools.cc:512-519)
  const double g = 0.57735026918962573;
  const double qp[4][2] = {{-g, -g}, {g, -g}, {g, g}, {-g, g}};
  const double jx = 0.5 * dx, jy = 0.5 * dy;
  FemGerms W;
  for (int q = 0; q < 4; ++q) {
    const double x = qp[q][0], y = qp[q][1];
    const double v[4] = {(1 - x) * (1 - y) / 4., (1 + x) * (1 - y) / 4., (1 + x) * (1 + y) / 4.,
                         (1 - x) * (1 + y) / 4.};
    const double ddx[4] = {-(1 - y) / 4., (1 - y) / 4., (1 + y) / 4., -(1 + y) / 4.};
    const double ddy[4] = {-(1 - x) / 4, -(1 + x) / 4, (1 + x) / 4, (1 - x) / 4};
    for (int k = 0; k < 4; ++k) {
      W.val[q][k] = v[k];
      W.gx[q][k] = ddx[k] / jx;
      W.gy[q][k] = ddy[k] / jy;
    }
    W.JxW[q] = jx * jy * 1.0;
  }
  return W;
}

int fem_allocate(FemState &S, int Mx, int My, int periodicity) {
  const int nex = (periodicity & 1) ? Mx : Mx - 1, ney = (periodicity & 2) ? My : My - 1;
  if (S.J && S.N == Mx * My && S.nex == nex && S.ney == ney) return 0;
  fem_free(S);
  S.nex = nex;
  S.ney = ney;
  S.Ne = nex * ney;
  S.N = Mx * My;
  const size_t Q = 4 * (size_t)S.Ne, N = S.N;
  int bad = alloc(&S.C.H, Q) | alloc(&S.C.tauc, Q) | alloc(&S.C.tdu, Q) | alloc(&S.C.tdv, Q) | alloc(&S.C.B, Q) |
            alloc(&S.C.mask, Q) | alloc(&S.J, 36 * N) | alloc(&S.dinv, N) | alloc(&S.F, N) | alloc(&S.Ft, N) |
            alloc(&S.du, N) | alloc(&S.trial, N) | alloc(&S.vel0, N) | alloc(&S.r, N) | alloc(&S.z, N) | alloc(&S.p, N) |
            alloc(&S.q, N) | alloc(&S.cg, 1) | alloc(&S.sc, 1) | alloc(&S.zero_pivot, 1);
  if (bad) {
    fem_free(S);
    return 1;
  }
  return 0;
}

void fem_free(FemState &S) {
  void *ptrs[] = {S.C.H, S.C.tauc, S.C.tdu, S.C.tdv, S.C.B, S.C.mask, S.J, S.dinv, S.F, S.Ft,
                  S.du, S.trial, S.vel0, S.r, S.z, S.p, S.q, S.cg, S.sc, S.zero_pivot};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (S.cg_batch) cudaGraphExecDestroy(S.cg_batch);
  S = FemState{};
}

void launch_fem_coefficients(const Launch &L, const FemProblem &P, const FemState &S, const double *H,
                             const double *bed, const double *tauc, const double *srf, const double *enthalpy,
                             const double *z, int Mz, double icefree_thickness, double is_floating_thickness) {
  const FemGrid G = fem_grid(P);
  L.tick();
  k_fem_coefficients<<<blocks(L, S.Ne), NTF, 0, L.stream>>>(G, P.c, P.W, S.C, H, bed, tauc, srf, enthalpy, z, Mz,
                                                            icefree_thickness, is_floating_thickness);
}

void launch_fem_residual(const Launch &L, const FemProblem &P, const FemState &S, const double2 *vel, double2 *F,
                         bool jacobian, const uint8_t *bc, const double2 *bcv) {
  const FemGrid G = fem_grid(P);
  L.tick();
  if (jacobian)
    k_fem_node<true><<<blocks(L, S.N), NTF, 0, L.stream>>>(P, G, S.C, vel, bc, bcv, F, S.J, S.dinv, S.zero_pivot,
                                                           S.sc, L.partials, L.ticket);
  else
    k_fem_node<false><<<blocks(L, S.N), NTF, 0, L.stream>>>(P, G, S.C, vel, bc, bcv, F, S.J, S.dinv,
                                                            S.zero_pivot, S.sc, L.partials, L.ticket);
}

void launch_fem_cg_init(const Launch &L, const FemProblem &P, const FemState &S, double rtol, int maxit) {
  L.tick();
  k_cg_init<<<blocks(L, S.N), NTF, 0, L.stream>>>(S.N, S.F, S.dinv, S.du, S.r, S.z, S.p, S.cg, rtol, maxit,
                                                  L.partials, L.ticket);
  (void)P;
}

void launch_fem_cg_iterations(const Launch &L, const FemProblem &P, const FemState &S, int n) {
  const FemGrid G = fem_grid(P);
  const int b = blocks(L, S.N);
  for (int it = 0; it < n; ++it) {
    L.tick(3);
    k_cg_apply<<<b, NTF, 0, L.stream>>>(G, S.J, S.p, S.q, S.cg, L.partials, L.ticket);
    k_cg_update<<<b, NTF, 0, L.stream>>>(S.N, S.dinv, S.p, S.q, S.du, S.r, S.z, S.cg, L.partials, L.ticket);
    k_cg_direction<<<b, NTF, 0, L.stream>>>(S.N, S.z, S.p, S.cg);
  }
}

void launch_fem_trial(const Launch &L, const FemState &S, const double2 *vel, double lambda) {
  L.tick();
  k_fem_trial<<<blocks(L, S.N), NTF, 0, L.stream>>>(S.N, vel, S.du, lambda, S.trial, S.sc, L.partials, L.ticket);
}

}  // namespace pism_gpu
