// ssa_internal.h — device buffers, solver state and kernel launchers of the B200
// SSAFD solver (shared by ssa_kernels.cu and ssa_capi.cu; not part of the C-ABI).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ssa_device.cuh"
#include "ssa_small_plan.h"
#include "ssa_state.h"

namespace pism_gpu {

// device fields of one grid (non-owning view)
struct Fields {
  const double *H, *srf, *bed, *tauc, *melange, *gl_mask, *enthalpy, *fracture;
  const double2 *bcv;
  const int8_t *mask;
  const uint8_t *bc;
  double2 *taud, *rhs, *hardness, *nuH, *vel;
  double *beta;
  uint32_t *flags;
  double nu_bedrock;
};

// Krylov work vectors (BiCGStab)
struct Krylov {
  double2 *r, *rhat, *p, *v, *s, *t, *phat, *shat;
  double4 *dinv;
  KState *st;
};

// Restarted flexible GMRES(m) (right preconditioning): Arnoldi basis V[0..m], the
// preconditioned directions Z[0..m-1] and the small dense state on the device
constexpr int GM_MAXM = 30;   // largest restart length (PETSc's default is 30)
struct GState {
  double H[GM_MAXM + 1][GM_MAXM];   // Hessenberg matrix, rotated into R in place
  double cs[GM_MAXM], sn[GM_MAXM];  // Givens rotations
  double g[GM_MAXM + 1];            // rotated right-hand side: |g[j+1]| = residual norm
  double y[GM_MAXM];
  double bnorm, hnext, scale0;
  int m, cols, cols_upd, need_update, restart;
};
struct Gmres {
  double2 *V, *Z;   // (m + 1) x N and m x N
  double *partials; // blocks x 32
  GState *gs;
  KState *st;       // done / status / iter / maxit / rtol shared with the multigrid early exit
  int m;
};

// FP32 work vectors of the inner solve of the mixed-precision path
struct Krylov32 {
  float2 *rhs, *r, *rhat, *p, *v, *t, *phat, *shat, *d;   // s = r - alpha v is never stored
  KState *st;
};

struct Launch {
  cudaStream_t stream;
  int max_blocks;        // resident blocks (SM count x blocks per SM)
  double *partials;      // per-block partial sums (>= max_blocks * 8)
  unsigned *ticket;      // last-block ticket, kept at 0 between kernels
  long long *count;      // kernel-launch counter (may be null)
  void tick(int n = 1) const {
    if (count) *count += n;
  }
};

// ---- aggregation multigrid (ssa_mg.cu) ----
constexpr int MG_MAX_LEVELS = 16;
constexpr int MG_COARSE_DIM = 4;                 // the coarsest level has <= 4 x 4 cells
constexpr int MG_MAX_COARSE_CELLS = MG_COARSE_DIM * MG_COARSE_DIM;
constexpr int MG_CTA_CELLS = 4096;               // levels this small are cycled by one thread-block cluster
constexpr int MG_CTA_CELLS_WIDE = 16384;         // ... with mg_small_kernel 2

struct MGLevel {
  int Mx = 0, My = 0, N = 0;
  int ax = 1, ay = 1;                            // aggregation factors towards the next level
  float4 *A = nullptr;                           // 9 stencil blocks x N (block b of cell k at b*N+k)
  float4 *dinv = nullptr;                        // inverse 2x2 diagonal blocks
  float2 *b = nullptr, *x = nullptr;
};

struct MGHierarchy {
  int nlev = 0;                                  // coarse levels (level 1 .. nlev)
  int fine_ax = 1, fine_ay = 1;                  // aggregation of the fine grid
  MGLevel lev[MG_MAX_LEVELS];
  int small_first = 0;                           // first level cycled by the cluster
  int small_first_wide = 0;                      // the same with mg_small_kernel 2
  int small_smem = 0;                            // its per-CTA staging buffer (bytes)
  bool small_dsmem = false;                      // the small levels fit the cluster's shared memory
  int small_kernel = 0;                          // mg_small_kernel of the configuration
  int apply_kernel = 2;                          // mixed_apply_kernel of the configuration
  SmallPlan small_plan{};                        // their split over the cluster's CTAs
  void *small_plan_dev = nullptr;                // device copy of small_plan
  float omega = 0.9f;                            // damping of the block-Jacobi smoother
  float correction = 1.2f;                       // scaling of the coarse-grid correction
  int post_blocks = 0;                           // grid cap of the coarse post-smoothing (0: none)
  double *cinv = nullptr;                        // dense inverse of the coarsest operator (transposed)
  int *singular = nullptr;
  float2 *nuHf = nullptr;                        // FP32 copies of the fine nu*H, beta, D^-1
  float *betaf = nullptr;
  float4 *dinvf = nullptr;
  void *views = nullptr;                         // device copy of the level views
};

int mg_plan(int Mx, int My, MGHierarchy &H);
int mg_allocate(MGHierarchy &H, int fine_cells);
void mg_free(MGHierarchy &H);

// Line block-Jacobi preconditioner.  Per cell, after line_setup: P = the inverse pivot
// block, F = -P L (forward multiplier), G = P U (backward multiplier) of the block LU
// factorisation of each grid line's 2 x 2-block tridiagonal part.
struct LinePC {
  double4 *P = nullptr, *F = nullptr, *G = nullptr;
};

void launch_convert_masks(const Launch &L, int N, const double *mask, const double *bc_mask, int8_t *mask_i,
                          uint8_t *bc_i);
void launch_prepare(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, int periodicity,
                    const Fields &f);
void launch_hardness(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const Fields &f, int Mz,
                     const double *z);
void launch_nuH(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const Fields &f, double reg,
                double underrelax, bool with_norm, double *norm_out);
void launch_apply(const Launch &L, const GridDev &g, const Fields &f, const double2 *x, double2 *y);
void launch_diag_setup(const Launch &L, const GridDev &g, const Fields &f, double4 *dinv, int *zero_diag_cell);
void launch_bicg_init(const Launch &L, const GridDev &g, const Fields &f, const Krylov &K, const double2 *b,
                      const double2 *x);
void launch_bicg_iteration(const Launch &L, const GridDev &g, const Fields &f, const Krylov &K, double2 *x,
                           const MGHierarchy *mg, const LinePC *line);
// FGMRES: r0 = b - A x into V0 (init) / after a restart; one Arnoldi step j; the end of a cycle
void launch_gmres_residual(const Launch &L, const GridDev &g, const Fields &f, const Gmres &G, const double2 *b,
                           const double2 *x, int init);
void launch_gmres_step(const Launch &L, const GridDev &g, const Fields &f, const Gmres &G, const double4 *dinv,
                       const MGHierarchy *mg, const LinePC *line, int j);
// the two halves of an Arnoldi step: z_j = M^-1 v_j, then w = A z_j orthogonalised
void launch_gmres_precondition(const Launch &L, const GridDev &g, const Fields &f, const Gmres &G,
                               const double4 *dinv, const MGHierarchy *mg, const LinePC *line, int j);
void launch_gmres_orthogonalize(const Launch &L, const GridDev &g, const Fields &f, const Gmres &G, int j);
// ad = A d; gamma = (r, ad) / (ad, ad); z += gamma d (skipped once st->done)
void launch_pc_line_search(const Launch &L, const GridDev &g, const Fields &f, const double2 *r, const double2 *d,
                           double2 *ad, double *gamma, double2 *z, const KState *st);
// r = v - A z (FP64), skipped once st->done
void launch_pc_residual(const Launch &L, const GridDev &g, const Fields &f, const double2 *v, const double2 *z,
                        double2 *r, const KState *st);
void launch_gmres_update(const Launch &L, const GridDev &g, const Gmres &G, double2 *x);
void mg_setup(const Launch &L, const GridDev &g, const Fields &f, const double4 *dinv0, MGHierarchy &H);
void mg_setup_fine(const Launch &L, const GridDev &g, const Fields &f, const double4 *dinv0, MGHierarchy &H);
void mg_setup_coarse(const Launch &L, const GridDev &g, const Fields &f, MGHierarchy &H);
void mg_vcycle(const Launch &L, const GridDev &g, const Fields &f, const MGHierarchy &H, const double2 *b,
               double2 *z, KState *st);
void mg_vcycle(const Launch &L, const GridDev &g, const Fields &f, const MGHierarchy &H, const float2 *b, float2 *z,
               KState *st);
// the V-cycle with right-hand side s = r - st->alpha v, formed on the fly (BiCGStab's s)
void mg_vcycle_s(const Launch &L, const GridDev &g, const Fields &f, const MGHierarchy &H, const float2 *r,
                 const float2 *v, float2 *z, KState *st);
// the FP32 V-cycles of BiCGStab with the operator apply that follows each fused into the
// fine-level pass: z = M^-1 b, then y = A z handed to the epilogue (ssa_krylov32.cuh)
struct EpiV;
struct EpiT;
void mg_vcycle_apply(const Launch &L, const GridDev &g, const Fields &f, const MGHierarchy &H, const float2 *b,
                     float2 *z, const EpiV &e);
void mg_vcycle_s_apply(const Launch &L, const GridDev &g, const Fields &f, const MGHierarchy &H, const float2 *r,
                       const float2 *v, float2 *z, const EpiT &e);
// ---- the consumers of the SSA velocity (ssa_column.cu, ssa_transport.cu) ----
void launch_mass_continuity(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const Fields &f,
                            double dt, double icefree_thickness, double is_floating_thickness, const double *cmb,
                            const double *bmr, const double *area, double *Hnew, double *fdiv, double *mask_new,
                            double *surface_new, double *totals);
// ---- strain rates, 2-D stresses and eigen-calving (ssa_calving.cu) ----
void launch_strain_rates(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const double2 *vel,
                         const int8_t *mask, double *edot, double *stress);
void launch_mask_from_doubles(const Launch &L, int N, const double *in, int8_t *a, int8_t *b);
void launch_eigen_calving_passes(const Launch &L, const GridDev &g, const double2 *vel, double K, double dt,
                                 double *H, double *Href, double *loss, int8_t *m0, int8_t *live);
void launch_tongue_sweep(const Launch &L, const GridDev &g, const int8_t *m0, int8_t *live, int *changed);
void launch_eigen_calving_finish(const Launch &L, int N, const int8_t *m0, const int8_t *live, double *H,
                                 double *mask_out);
void launch_eigen_calving_rates(const Launch &L, const GridDev &g, const double2 *vel, const int8_t *mask, double K,
                                double *out, unsigned long long *rmax);
constexpr int SB3D_MAX_LEVELS = 800;   // the column kernel's shared-memory tile holds 32 columns
int stress_balance_3d_prepare(int Mz);
void launch_stress_balance_3d(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, int Mz,
                              const Fields &f, const double *z, const double *bmr, double *u3, double *v3,
                              double *w3, double *sigma);
// ---- line block-Jacobi preconditioner (ssa_line.cu) ----
void line_setup(const Launch &L, const GridDev &g, const Fields &f, const double4 *dinv, const LinePC &lp);
void line_apply(const Launch &L, const GridDev &g, const LinePC &lp, const double2 *b, double2 *z, const KState *st);
// z = M^-1 r with block Jacobi (dinv), the multigrid cycle (mg) or the line solve (line)
void launch_pc_apply(const Launch &L, const GridDev &g, const Fields &f, const double4 *dinv, const MGHierarchy *mg,
                     const LinePC *line, const double2 *r, double2 *z);

// ---- device-side control of the Picard loop (ssa_control.cu; state and decisions in
// ssa_state.h) ----
void launch_picard_start(const Launch &L, PState *P);
// a Picard pass begins: zero-diagonal marker reset, the pass's KSP tolerance
void launch_picard_begin(const Launch &L, PState *P, const PicardConst &c, int *zero_diag_cell);
// FP64 BiCGStab inside the graph: its state from the pass's tolerance; its outcome
void launch_ksp_begin(const Launch &L, KState *st, const PState *P, int maxit);
void launch_ksp_end(const Launch &L, PState *P, const KState *st, int body_iters);
// the end of one refinement step of the mixed-precision solve (go = apply its correction)
void launch_refine_end(const Launch &L, PState *P, const KState *st, int max_refine);
void launch_picard_after_solve(const Launch &L, PState *P, const int *zero_diag_cell);
void launch_picard_test(const Launch &L, PState *P, const double *norm2, const PicardConst &c);
// a conditional node's value from a flag: flag != 0 (or == 0 when negate)
void launch_flag_condition(const Launch &L, cudaGraphConditionalHandle cond, const int *flag, bool negate);
// launch_mixed_init with the outer tolerance read from the device
void launch_mixed_init_dev(const Launch &L, int N, const Krylov32 &K, const double *res2, const double *outer_rtol,
                           double inner_min, int maxit);

// the loop condition of a graph-resident Krylov loop: continue while st->done is 0
void launch_loop_condition(const Launch &L, cudaGraphConditionalHandle cond, const KState *st);

// the start of an inner FP32 solve; the outer test and the inner tolerance are taken on the
// device from res2 = {||b - A x||^2, ||b||^2} (launch_residual32)
void launch_mixed_init(const Launch &L, int N, const Krylov32 &K, const double *res2, double outer_rtol,
                       double inner_min, int maxit);
void launch_mixed_iteration(const Launch &L, const GridDev &g, const Fields &f, const MGHierarchy &H,
                            const Krylov32 &K);
// r32 = (float) (b - A x) with FP64 arithmetic; out2 = {||b - A x||^2, ||b||^2}
void launch_residual32(const Launch &L, const GridDev &g, const Fields &f, const double2 *b, const double2 *x,
                       float2 *r32, double *out2);
// x += d
void launch_axpy32(const Launch &L, int N, const float2 *d, double2 *x);
void launch_bfrict(const Launch &L, int N, const pism_gpu_ssa_config &c, const Fields &f, double *out);
void launch_scale(const Launch &L, int n, double a, double *x);

}  // namespace pism_gpu
