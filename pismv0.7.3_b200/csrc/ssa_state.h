// ssa_state.h — the solver scalars the device keeps (Krylov state, the whole-solve graph's
// Picard state) and the Picard-loop decisions on them, as plain C++ so that the host
// compiler can check the decisions too.  Included by ssa_internal.h.
#pragma once

#if defined(__CUDACC__)
#define PISM_HD __host__ __device__ __forceinline__
#else
#define PISM_HD inline
#endif

#include <climits>
#include <cmath>

#include "../../include/pism_ssa_gpu.h"

namespace pism_gpu {

// Krylov status codes written by the device (KSPConvergedReason analogues); KSP_STALLED: a
// kernel's bounded wait for data staged by the bulk-copy engine gave up (the solve stops
// rather than go on with a preconditioner or operator that may have used late data)
enum : int { KSP_OK = 0, KSP_MAXIT = -3, KSP_BREAKDOWN = -5, KSP_NAN = -7, KSP_STALLED = -11 };
constexpr int KSP_OUTER_DONE = 1;   // mixed precision: the outer residual already meets the tolerance

// scalars of one Krylov solve, owned by the device
struct KState {
  double rho, alpha, omega, beta;
  double rnorm2, bnorm2, rnorm0, rtol;
  double outer_r2, outer_b2;   // the FP64 outer residual of a mixed-precision refinement step
  int iter, maxit, done, status;
};

// The state a whole-solve graph keeps on the device: the decisions of the host loop
// (SSAFD::picard_manager, SSAFD.cc:962-1119, and the refinement loop of the mixed-precision
// solve) taken by single-thread kernels, and the counts the host reads back once.
struct PState {
  double rtol;          // KSP tolerance of the current Picard iteration
  double last_change;   // relative nu*H change of the previous iteration
  double norm, change;  // the last Picard test's norms
  double final_res;     // relative residual of the last linear solve
  int k;                // Picard tests taken (= Picard iterations)
  int passes;           // Picard loop passes
  int done, status;     // status: a PISM_GPU_SSA_* code once done
  int zd_cell;          // the zero-diagonal cell, when status is EZERODIAG
  int ksp_its, ksp_status, ksp_total;
  int refine, refine_done, go, go_count, refine_steps, refine_passes;
  long long inner_passes;   // passes of the innermost Krylov loop body
  double coarse_change;     // relative nu*H changes summed since the coarse levels were built
  int rebuild;              // this pass rebuilds the multigrid coarse levels
  int rebuilds;             // coarse-level builds of the solve
};
struct PicardConst {
  double ksp_rtol, ksp_rtol_max, ksp_rtol_factor, picard_rtol;
  int adaptive, max_iterations;
  double mg_rebuild_rtol;   // lagged coarse levels: rebuild once the summed change reaches this (0: always)
};

// ---- the decisions (the host loop's, in the same double arithmetic) ----

// Whether a Picard pass rebuilds the multigrid coarse levels (their Galerkin operators and
// the coarsest inverse) from the current nu*H: always on the first pass of a solve and
// without lagging; with lagging once the relative nu*H changes summed since the last build
// (a bound on the relative change since then) reach mg_rebuild_rtol.  The fine level and
// the Krylov operator always use the current nu*H; a lagged coarse level only changes how
// fast the preconditioned iteration converges, not the tolerance it meets.
PISM_HD bool mg_rebuild_due(double &coarse_change, bool first, double mg_rebuild_rtol) {
  const bool due = first || !(mg_rebuild_rtol > 0.0) || coarse_change >= mg_rebuild_rtol;
  if (due) coarse_change = 0.0;
  return due;
}

// after a Picard test: the change since the coarse levels were built grows by this one
PISM_HD void mg_change_add(double &coarse_change, double norm, double change) {
  if (norm > 0.0 && std::isfinite(norm) && std::isfinite(change)) coarse_change += change / norm;
}

PISM_HD void picard_start(PState &P) {
  P = PState{};
  P.last_change = 1.0;
}

// a Picard pass begins: the KSP tolerance of inexact Picard (picard_manager's rtol)
PISM_HD void picard_begin(PState &P, const PicardConst &c) {
  P.rebuild = mg_rebuild_due(P.coarse_change, P.passes == 0, c.mg_rebuild_rtol) ? 1 : 0;
  P.rebuilds += P.rebuild;
  double rtol = c.ksp_rtol;
  if (c.adaptive && P.last_change >= 2.0 * c.picard_rtol)
    rtol = fmin(c.ksp_rtol_max, fmax(c.ksp_rtol, c.ksp_rtol_factor * P.last_change));
  P.rtol = rtol;
  P.passes += 1;
  P.ksp_its = 0;
  P.ksp_status = KSP_OK;
  P.refine = 0;
  P.refine_done = 0;
  P.go = 0;
}

PISM_HD void ksp_begin(KState &st, const PState &P, int maxit) {
  st = KState{};
  st.rtol = P.rtol;
  st.maxit = maxit;
}

PISM_HD void ksp_end(PState &P, const KState &st, int body_iters) {
  P.ksp_its = st.iter;
  P.ksp_status = st.status;
  P.final_res = st.bnorm2 > 0 ? sqrt(st.rnorm2 / st.bnorm2) : sqrt(st.rnorm2);
  P.inner_passes += (st.iter + body_iters - 1) / body_iters;
}

// the refinement loop body of linear_solve_mixed after an inner solve
PISM_HD void refine_end(PState &P, const KState &st, int max_refine) {
  const double rn = sqrt(st.outer_r2), bn = sqrt(st.outer_b2);
  P.final_res = bn > 0 ? rn / bn : rn;
  P.inner_passes += st.iter;
  P.refine_passes += 1;
  int stop = 0, status = KSP_OK;
  if (!std::isfinite(rn)) {
    status = KSP_NAN;
    stop = 1;
  } else if (st.status == KSP_OUTER_DONE) {
    stop = 1;
  } else if (P.refine >= max_refine) {
    status = KSP_MAXIT;
    stop = 1;
  } else {
    P.ksp_its += st.iter;
    P.refine_steps += 1;
    if (st.status == KSP_NAN || st.status == KSP_STALLED) {
      status = st.status;
      stop = 1;
    } else if (st.iter == 0) {
      status = KSP_BREAKDOWN;
      stop = 1;
    }
  }
  if (stop) {
    P.refine_done = 1;
    P.ksp_status = status;
    P.go = 0;
  } else {
    P.refine += 1;
    P.go = 1;
    P.go_count += 1;
  }
}

// picard_manager after a linear solve: the zero-diagonal and KSP checks
PISM_HD void picard_after_solve(PState &P, int zero_diag_cell) {
  P.ksp_total += P.ksp_its;
  if (zero_diag_cell != INT_MAX) {
    P.zd_cell = zero_diag_cell;
    P.status = PISM_GPU_SSA_EZERODIAG;
    P.done = 1;
  } else if (P.ksp_status != KSP_OK) {
    P.status = PISM_GPU_SSA_EKSP;
    P.done = 1;
  }
}

// the Picard test, SSAFD.cc:1084, with inexact Picard's "last solve to ksp_rtol" rule
PISM_HD void picard_test(PState &P, double norm, double change, const PicardConst &c) {
  P.k += 1;
  P.norm = norm;
  P.change = change;
  mg_change_add(P.coarse_change, norm, change);
  if (!std::isfinite(norm) || !std::isfinite(change)) {
    P.status = PISM_GPU_SSA_ENAN;
    P.done = 1;
    return;
  }
  if (norm == 0 || (change / norm < c.picard_rtol && P.rtol <= c.ksp_rtol)) {
    P.status = PISM_GPU_SSA_OK;
    P.done = 1;
    return;
  }
  P.last_change = norm > 0 ? change / norm : 0.0;
  if (P.k >= c.max_iterations) {
    P.status = PISM_GPU_SSA_EPICARD;
    P.done = 1;
  }
}

}  // namespace pism_gpu
