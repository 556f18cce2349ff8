// ssafd_cpu.cc — TEST INFRASTRUCTURE ONLY (CPU oracle / timed CPU baseline, never the product).
//
// A native restatement of the reference's SSAFD Picard loop on the host cores, the way a
// PETSc build of PISM runs it: per Picard iteration nu*H on the staggered grid
// (SSAFD::compute_nuH_staggered, src/base/stressbalance/ssa/SSAFD.cc:1359-1421), the basal
// drag (basal_resistance.cc:46-50, 154-163; SSAFD.cc:744-763), the 18-column matrix
// assembly (SSAFD::assemble_matrix, SSAFD.cc:496-811, here without the calving-front
// weights), the KSP solve (ksp_cpu.cc: PETSc's GMRES(30) + block Jacobi / ILU(0), one block
// per rank, in PETSc's rank-major unknown order), the under-relaxation (SSAFD.cc:1061-1064),
// the nu*H norms over the ghosted arrays (SSAFD.cc:1170-1189) and the stopping test
// (SSAFD.cc:1084).  Driving stress, right-hand side and hardness (once per solve) come from
// the Python oracle.  The arithmetic follows oracle/ssafd_oracle.py term by term (the CPU
// suite checks the two against each other); the unknowns' order is the oracle's
// 2 * (i * My + j) + component, mapped to PETSc's by `perm`.
//
// C ABI (ctypes): ssafd_cpu_picard(...).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include <omp.h>

extern "C" int ksp_gmres_bjacobi_ilu0(int n, const int *rowptr, const int *col, const double *val, int nblocks,
                                      const int *block_start, const double *b, double *x, double rtol, double abstol,
                                      double dtol, int maxit, int restart, int nthreads, int *its, double *rnorm_out,
                                      double *rnorm0_out);

namespace {

// parameters of the path, in this order in the `par` array of ssafd_cpu_picard
struct Par {
  double dx, dy;
  double glen_n, enhancement, schoof_reg;     // Glen exponent, enhancement factor, (v_S / L_S)^2
  double hmin, nu_ext;                        // strength extension: H_min, constant nu
  double plastic_reg, pseudo, q, uthreshold, tauc_scale;   // drag
  double beta_ice_free, scaling;              // ice-free-land drag, Dirichlet diagonal
};

inline int wrap(int a, int M) { return a < 0 ? a + M : (a >= M ? a - M : a); }

// mask predicates (src/base/util/Mask.hh:28-65)
inline bool grounded_ice(int m) { return m == 2; }
inline bool ice_free_land(int m) { return m == 0; }

struct Grid {
  int Mx, My;
  int at(int i, int j) const { return wrap(i, Mx) * My + wrap(j, My); }
};

// FlowLaw::effective_viscosity (flowlaws.hh:100-112) with secondInvariant_2D (flowlaws.hh:36-39)
inline double eff_visc(const Par &p, double B, double u_x, double u_y, double v_x, double v_y) {
  const double gamma = 0.5 * (u_x * u_x + v_y * v_y + (u_x + v_y) * (u_x + v_y) + 0.5 * ((u_y + v_x) * (u_y + v_x)));
  return 0.5 * B * std::pow(p.schoof_reg + gamma, (1.0 - p.glen_n) / (2.0 * p.glen_n));
}

// SSAFD::compute_nuH_staggered, SSAFD.cc:1359-1421
void compute_nuH(const Grid &g, const Par &p, const double *H, const double *hard, const double *vel, double reg,
                 double *nuH) {
  const double scal = 1.0 / std::pow(p.enhancement, 1.0 / p.glen_n);
  const double notional = p.nu_ext * p.hmin;
  const double dx = p.dx, dy = p.dy;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < g.Mx; ++i)
    for (int j = 0; j < g.My; ++j) {
      const int k = i * g.My + j;
      auto U = [&](int di, int dj) { return vel[2 * g.at(i + di, j + dj)]; };
      auto V = [&](int di, int dj) { return vel[2 * g.at(i + di, j + dj) + 1]; };
      for (int o = 0; o < 2; ++o) {
        const int oi = 1 - o, oj = o;
        const double Hf = 0.5 * (H[k] + H[g.at(i + oi, j + oj)]);
        double u_x, u_y, v_x, v_y;
        if (o == 0) {
          u_x = (U(1, 0) - U(0, 0)) / dx;
          u_y = (U(0, 1) + U(1, 1) - U(0, -1) - U(1, -1)) / (4 * dy);
          v_x = (V(1, 0) - V(0, 0)) / dx;
          v_y = (V(0, 1) + V(1, 1) - V(0, -1) - V(1, -1)) / (4 * dy);
        } else {
          u_x = (U(1, 0) + U(1, 1) - U(-1, 0) - U(-1, 1)) / (4 * dx);
          u_y = (U(0, 1) - U(0, 0)) / dy;
          v_x = (V(1, 0) + V(1, 1) - V(-1, 0) - V(-1, 1)) / (4 * dx);
          v_y = (V(0, 1) - V(0, 0)) / dy;
        }
        double r = eff_visc(p, hard[2 * k + o], u_x, u_y, v_x, v_y) * Hf;
        r = r * scal;
        r = r + reg;
        nuH[2 * k + o] = Hf < p.hmin ? notional : r;
      }
    }
}

// IceBasalResistance{Plastic,PseudoPlastic}Law::drag, basal_resistance.cc:46-50, 154-163
inline double drag(const Par &p, double tauc, double u, double v) {
  const double magreg2 = p.plastic_reg * p.plastic_reg + u * u + v * v;
  if (p.pseudo == 0.0) return tauc / std::sqrt(magreg2);
  if (p.tauc_scale > 0.0)
    return (tauc / std::pow(p.tauc_scale, p.q)) * std::pow(magreg2, 0.5 * (p.q - 1)) * std::pow(p.uthreshold, -p.q);
  return tauc * std::pow(magreg2, 0.5 * (p.q - 1)) * std::pow(p.uthreshold, -p.q);
}

// the basal drag coefficient on the diagonal, SSAFD.cc:744-763
void beta_field(const Grid &g, const Par &p, const int *mask, const double *tauc, const double *vel, double *beta) {
  const int N = g.Mx * g.My;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < N; ++k) {
    const int m = mask[k];
    beta[k] = grounded_ice(m) ? drag(p, tauc[k], vel[2 * k], vel[2 * k + 1])
                              : (ice_free_land(m) ? p.beta_ice_free : 0.0);
  }
}

// (I, J) offsets and component of the 18 stencil entries (SSAFD.cc:710-737)
const int DI[18] = {-1, 0, 1, -1, 0, 1, -1, 0, 1, -1, 0, 1, -1, 0, 1, -1, 0, 1};
const int DJ[18] = {1, 1, 1, 0, 0, 0, -1, -1, -1, 1, 1, 1, 0, 0, 0, -1, -1, -1};
const int CC[18] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1};

// the eq1 (component 0) or eq2 (component 1) coefficients of one cell, SSAFD.cc:594-737,
// with every calving-front weight 1 (no CFBC)
void coefficients(const Grid &g, const Par &p, const double *nuH, const double *beta, int i, int j, int comp,
                  double e[18]) {
  const double c_w = nuH[2 * g.at(i - 1, j)], c_e = nuH[2 * g.at(i, j)];
  const double c_s = nuH[2 * g.at(i, j - 1) + 1], c_n = nuH[2 * g.at(i, j) + 1];
  const double aMn = 1, aPn = 1, aMM = 1, aPP = 1, aMs = 1, aPs = 1;
  const double bPw = 1, bPP = 1, bPe = 1, bMw = 1, bMM = 1, bMe = 1;
  const double dx2 = p.dx * p.dx, dy2 = p.dy * p.dy, d4 = 4 * p.dx * p.dy, d2 = 2 * p.dx * p.dy;
  if (comp == 0) {
    e[0] = 0; e[1] = -c_n * bPP / dy2; e[2] = 0;
    e[3] = -4 * c_w * aMM / dx2;
    e[4] = (c_n * bPP + c_s * bMM) / dy2 + (4 * c_e * aPP + 4 * c_w * aMM) / dx2;
    e[5] = -4 * c_e * aPP / dx2;
    e[6] = 0; e[7] = -c_s * bMM / dy2; e[8] = 0;
    e[9] = c_w * aMM * bPw / d2 + c_n * aMn * bPP / d4;
    e[10] = (c_n * aPn * bPP - c_n * aMn * bPP) / d4 + (c_w * aMM * bPP - c_e * aPP * bPP) / d2;
    e[11] = -c_e * aPP * bPe / d2 - c_n * aPn * bPP / d4;
    e[12] = (c_w * aMM * bMw - c_w * aMM * bPw) / d2 + (c_n * aMM * bPP - c_s * aMM * bMM) / d4;
    e[13] = (c_n * aPP * bPP - c_n * aMM * bPP - c_s * aPP * bMM + c_s * aMM * bMM) / d4 +
            (c_e * aPP * bPP - c_w * aMM * bPP - c_e * aPP * bMM + c_w * aMM * bMM) / d2;
    e[14] = (c_e * aPP * bPe - c_e * aPP * bMe) / d2 + (c_s * aPP * bMM - c_n * aPP * bPP) / d4;
    e[15] = -c_w * aMM * bMw / d2 - c_s * aMs * bMM / d4;
    e[16] = (c_s * aMs * bMM - c_s * aPs * bMM) / d4 + (c_e * aPP * bMM - c_w * aMM * bMM) / d2;
    e[17] = c_e * aPP * bMe / d2 + c_s * aPs * bMM / d4;
    e[4] = e[4] + beta[i * g.My + j];
  } else {
    e[0] = c_w * aMM * bPw / d4 + c_n * aMn * bPP / d2;
    e[1] = (c_n * aPn * bPP - c_n * aMn * bPP) / d2 + (c_w * aMM * bPP - c_e * aPP * bPP) / d4;
    e[2] = -c_e * aPP * bPe / d4 - c_n * aPn * bPP / d2;
    e[3] = (c_w * aMM * bMw - c_w * aMM * bPw) / d4 + (c_n * aMM * bPP - c_s * aMM * bMM) / d2;
    e[4] = (c_n * aPP * bPP - c_n * aMM * bPP - c_s * aPP * bMM + c_s * aMM * bMM) / d2 +
           (c_e * aPP * bPP - c_w * aMM * bPP - c_e * aPP * bMM + c_w * aMM * bMM) / d4;
    e[5] = (c_e * aPP * bPe - c_e * aPP * bMe) / d4 + (c_s * aPP * bMM - c_n * aPP * bPP) / d2;
    e[6] = -c_w * aMM * bMw / d4 - c_s * aMs * bMM / d2;
    e[7] = (c_s * aMs * bMM - c_s * aPs * bMM) / d2 + (c_e * aPP * bMM - c_w * aMM * bMM) / d4;
    e[8] = c_e * aPP * bMe / d4 + c_s * aPs * bMM / d2;
    e[9] = 0; e[10] = -4 * c_n * bPP / dy2; e[11] = 0;
    e[12] = -c_w * aMM / dx2;
    e[13] = (4 * c_n * bPP + 4 * c_s * bMM) / dy2 + (c_e * aPP + c_w * aMM) / dx2;
    e[14] = -c_e * aPP / dx2;
    e[15] = 0; e[16] = -4 * c_s * bMM / dy2; e[17] = 0;
    e[13] = e[13] + beta[i * g.My + j];
  }
}

// The assembled matrix in PETSc's order: 18 entries per row, columns ascending (the
// DMDA-preallocated pattern keeps its explicit zeros).  The pattern is built once; the
// values every Picard iteration (MatSetValuesStencil).
struct Assembly {
  int n = 0;
  std::vector<int> rowptr, col, src;   // src: stencil slot m of each stored entry
  std::vector<int> cell, comp;         // per PETSc row: the oracle's cell and component
  std::vector<double> val;
  void pattern(const Grid &g, const int *perm, const std::vector<int> &inv) {
    n = 2 * g.Mx * g.My;
    rowptr.resize(n + 1);
    col.resize((size_t)18 * n);
    src.resize((size_t)18 * n);
    val.resize((size_t)18 * n);
    cell.resize(n);
    comp.resize(n);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; ++r) {
      const int q = perm[r], c = q / 2, i = c / g.My, j = c % g.My;
      cell[r] = c;
      comp[r] = q % 2;
      rowptr[r + 1] = 18 * (r + 1);
      std::pair<int, int> e[18];
      for (int m = 0; m < 18; ++m) e[m] = {inv[2 * g.at(i + DI[m], j + DJ[m]) + CC[m]], m};
      std::sort(e, e + 18);
      for (int m = 0; m < 18; ++m) {
        col[(size_t)18 * r + m] = e[m].first;
        src[(size_t)18 * r + m] = e[m].second;
      }
    }
    rowptr[0] = 0;
  }
  // values at nu*H, beta; rows of Dirichlet cells (bc[cell] != 0) hold the scaled identity
  void values(const Grid &g, const Par &p, const double *nuH, const double *beta, const int *bc) {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; ++r) {
      const int c = cell[r], i = c / g.My, j = c % g.My, cp = comp[r];
      double e[18];
      coefficients(g, p, nuH, beta, i, j, cp, e);
      const bool diag_only = bc && bc[c] != 0;
      for (int m = 0; m < 18; ++m) {
        const int s = src[(size_t)18 * r + m];
        double v = diag_only ? 0.0 : e[s];
        if (diag_only && s == (cp == 0 ? 4 : 13)) v += p.scaling;
        val[(size_t)18 * r + m] = v;
      }
    }
  }
};

// SSAFD::compute_nuH_norm, SSAFD.cc:1170-1189: L1 over the ghosted local vectors (every
// edge cell counted once more per periodic ghost copy), times the cell area
void nuH_norms(const Grid &g, const Par &p, const double *nuH, const double *old, double *norm, double *change) {
  double a0 = 0, a1 = 0, d0 = 0, d1 = 0;
#pragma omp parallel for schedule(static) reduction(+ : a0, a1, d0, d1)
  for (int i = 0; i < g.Mx; ++i) {
    const double wi = 1.0 + (i == 0) + (i == g.Mx - 1);
    for (int j = 0; j < g.My; ++j) {
      const double w = wi * (1.0 + (j == 0) + (j == g.My - 1));
      const int k = i * g.My + j;
      a0 += std::fabs(nuH[2 * k]) * w;
      a1 += std::fabs(nuH[2 * k + 1]) * w;
      d0 += std::fabs(old[2 * k] - nuH[2 * k]) * w;
      d1 += std::fabs(old[2 * k + 1] - nuH[2 * k + 1]) * w;
    }
  }
  const double area = p.dx * p.dy;
  a0 *= area; a1 *= area; d0 *= area; d1 *= area;
  *norm = std::sqrt(a0 * a0 + a1 * a1);
  *change = std::sqrt(d0 * d0 + d1 * d1);
}

}  // namespace

extern "C" {

// SSAFD::picard_manager (SSAFD.cc:962-1119) on the host cores.  vel (2N, the oracle's
// order) holds the initial guess and receives the last iterate.  par: the Par fields in
// order.  perm (2N): the oracle's unknown of each PETSc row; block_start (nranks + 1):
// PETSc's rank blocks.  Per iteration k < *picard_its the arrays ksp_its, t_nuH, t_asm,
// t_ksp, rel_change (each max_iterations long, may be NULL) get the KSP iterations, the
// seconds spent in nu*H + norms, drag + assembly and the KSP solve, and the relative nu*H
// change of the Picard test.  Returns 0 converged,
// 1 Picard limit reached, or the negative KSP reason of a failed solve.
int ssafd_cpu_picard(int Mx, int My, const double *par, const double *H, const int *mask, const double *tauc,
                     const double *hardness, const int *bc, const double *b, double *vel, const int *perm,
                     int nranks, const int *block_start, int nthreads, int max_iterations, double picard_rtol,
                     double ksp_rtol, int ksp_maxit, int restart, double reg, double underrelax, int *picard_its,
                     double *norm_out, double *change_out, int *ksp_its, double *t_nuH, double *t_asm,
                     double *t_ksp, double *rel_change) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Par p;
  std::memcpy(&p, par, sizeof(Par));
  const Grid g{Mx, My};
  const int N = Mx * My, n = 2 * N;
  std::vector<int> inv(n);
  for (int r = 0; r < n; ++r) inv[perm[r]] = r;
  Assembly A;
  A.pattern(g, perm, inv);
  std::vector<double> nuH(n), old(n), beta(N), bp(n), xp(n);
  for (int r = 0; r < n; ++r) bp[r] = b[perm[r]];
  double t0 = omp_get_wtime();
  compute_nuH(g, p, H, hardness, vel, reg, nuH.data());
  double t_pre = omp_get_wtime() - t0;
  *picard_its = 0;
  for (int k = 0; k < max_iterations; ++k) {
    t0 = omp_get_wtime();
    old = nuH;
    beta_field(g, p, mask, tauc, vel, beta.data());
    A.values(g, p, nuH.data(), beta.data(), bc);
    const double t1 = omp_get_wtime();
    for (int r = 0; r < n; ++r) xp[r] = vel[perm[r]];
    int its = 0;
    double rn = 0, rn0 = 0;
    const int reason = ksp_gmres_bjacobi_ilu0(n, A.rowptr.data(), A.col.data(), A.val.data(), nranks, block_start,
                                              bp.data(), xp.data(), ksp_rtol, 1e-50, 1e5, ksp_maxit, restart,
                                              nthreads, &its, &rn, &rn0);
    for (int r = 0; r < n; ++r) vel[perm[r]] = xp[r];
    const double t2 = omp_get_wtime();
    if (ksp_its) ksp_its[k] = its;
    if (reason < 0) {
      *picard_its = k;
      return reason;
    }
    compute_nuH(g, p, H, hardness, vel, reg, nuH.data());
    if (underrelax != 1.0)
      for (int q = 0; q < n; ++q) {
        nuH[q] = nuH[q] * underrelax;
        nuH[q] = nuH[q] + (1.0 - underrelax) * old[q];
      }
    double norm = 0, change = 0;
    nuH_norms(g, p, nuH.data(), old.data(), &norm, &change);
    const double t3 = omp_get_wtime();
    if (t_nuH) t_nuH[k] = (t3 - t2) + (k == 0 ? t_pre : 0.0);
    if (t_asm) t_asm[k] = t1 - t0;
    if (t_ksp) t_ksp[k] = t2 - t1;
    if (rel_change) rel_change[k] = norm > 0 ? change / norm : 0.0;
    *picard_its = k + 1;
    *norm_out = norm;
    *change_out = change;
    if (norm == 0 || change / norm < picard_rtol) return 0;
  }
  return 1;
}

}  // extern "C"
