// ssa_control.cu — device-side control of the Picard loop.
//
// A whole SSAFD solve (SSAFD::picard_manager, SSAFD.cc:962-1119, with its linear solves) can
// run as one CUDA graph whose conditional WHILE / IF nodes take their values from a PState
// in device memory.  These single-thread kernels make the decisions the host loop makes, in
// the same double arithmetic, so the graph takes the same path: the KSP tolerance of each
// Picard iteration (inexact Picard), the refinement steps of the mixed-precision solve, the
// zero-diagonal and KSP-failure checks and the Picard stopping test (SSAFD.cc:1084).
#include <climits>

#include "ssa_internal.h"

namespace pism_gpu {
namespace {

__global__ void k_picard_start(PState *P) {
  PState z{};
  z.last_change = 1.0;
  *P = z;
}

__global__ void k_picard_begin(PState *P, PicardConst c, int *zero_diag_cell) {
  *zero_diag_cell = INT_MAX;
  double rtol = c.ksp_rtol;
  if (c.adaptive && P->last_change >= 2.0 * c.picard_rtol)
    rtol = fmin(c.ksp_rtol_max, fmax(c.ksp_rtol, c.ksp_rtol_factor * P->last_change));
  P->rtol = rtol;
  P->passes += 1;
  P->ksp_its = 0;
  P->ksp_status = KSP_OK;
  P->refine = 0;
  P->refine_done = 0;
  P->go = 0;
}

__global__ void k_ksp_begin(KState *st, const PState *P, int maxit) {
  KState z{};
  z.rtol = P->rtol;
  z.maxit = maxit;
  *st = z;
}

__global__ void k_ksp_end(PState *P, const KState *st, int body_iters) {
  P->ksp_its = st->iter;
  P->ksp_status = st->status;
  P->final_res = st->bnorm2 > 0 ? sqrt(st->rnorm2 / st->bnorm2) : sqrt(st->rnorm2);
  P->inner_passes += (st->iter + body_iters - 1) / body_iters;
}

// the host's refinement loop body after an inner solve (linear_solve_mixed)
__global__ void k_refine_end(PState *P, const KState *st, int max_refine) {
  const double rn = sqrt(st->outer_r2), bn = sqrt(st->outer_b2);
  P->final_res = bn > 0 ? rn / bn : rn;
  P->inner_passes += st->iter;
  P->refine_passes += 1;
  int stop = 0, status = KSP_OK;
  if (!isfinite(rn)) {
    status = KSP_NAN;
    stop = 1;
  } else if (st->status == KSP_OUTER_DONE) {
    stop = 1;
  } else if (P->refine >= max_refine) {
    status = KSP_MAXIT;
    stop = 1;
  } else {
    P->ksp_its += st->iter;
    P->refine_steps += 1;
    if (st->status == KSP_NAN) {
      status = KSP_NAN;
      stop = 1;
    } else if (st->iter == 0) {
      status = KSP_BREAKDOWN;
      stop = 1;
    }
  }
  if (stop) {
    P->refine_done = 1;
    P->ksp_status = status;
    P->go = 0;
  } else {
    P->refine += 1;
    P->go = 1;
    P->go_count += 1;
  }
}

__global__ void k_picard_after_solve(PState *P, const int *zero_diag_cell) {
  P->ksp_total += P->ksp_its;
  if (*zero_diag_cell != INT_MAX) {
    P->zd_cell = *zero_diag_cell;
    P->status = PISM_GPU_SSA_EZERODIAG;
    P->done = 1;
  } else if (P->ksp_status != KSP_OK) {
    P->status = PISM_GPU_SSA_EKSP;
    P->done = 1;
  }
}

__global__ void k_picard_test(PState *P, const double *norm2, PicardConst c) {
  const double norm = norm2[0], change = norm2[1];
  P->k += 1;
  P->norm = norm;
  P->change = change;
  if (!isfinite(norm) || !isfinite(change)) {
    P->status = PISM_GPU_SSA_ENAN;
    P->done = 1;
    return;
  }
  if (norm == 0 || (change / norm < c.picard_rtol && P->rtol <= c.ksp_rtol)) {
    P->status = PISM_GPU_SSA_OK;
    P->done = 1;
    return;
  }
  P->last_change = norm > 0 ? change / norm : 0.0;
  if (P->k >= c.max_iterations) {
    P->status = PISM_GPU_SSA_EPICARD;
    P->done = 1;
  }
}

__global__ void k_flag_condition(cudaGraphConditionalHandle cond, const int *flag, int negate) {
  const bool on = (*flag != 0) != (negate != 0);
  cudaGraphSetConditional(cond, on ? 1u : 0u);
}

}  // namespace

void launch_picard_start(const Launch &L, PState *P) {
  L.tick();
  k_picard_start<<<1, 1, 0, L.stream>>>(P);
}
void launch_picard_begin(const Launch &L, PState *P, const PicardConst &c, int *zero_diag_cell) {
  L.tick();
  k_picard_begin<<<1, 1, 0, L.stream>>>(P, c, zero_diag_cell);
}
void launch_ksp_begin(const Launch &L, KState *st, const PState *P, int maxit) {
  L.tick();
  k_ksp_begin<<<1, 1, 0, L.stream>>>(st, P, maxit);
}
void launch_ksp_end(const Launch &L, PState *P, const KState *st, int body_iters) {
  L.tick();
  k_ksp_end<<<1, 1, 0, L.stream>>>(P, st, body_iters);
}
void launch_refine_end(const Launch &L, PState *P, const KState *st, int max_refine) {
  L.tick();
  k_refine_end<<<1, 1, 0, L.stream>>>(P, st, max_refine);
}
void launch_picard_after_solve(const Launch &L, PState *P, const int *zero_diag_cell) {
  L.tick();
  k_picard_after_solve<<<1, 1, 0, L.stream>>>(P, zero_diag_cell);
}
void launch_picard_test(const Launch &L, PState *P, const double *norm2, const PicardConst &c) {
  L.tick();
  k_picard_test<<<1, 1, 0, L.stream>>>(P, norm2, c);
}
void launch_flag_condition(const Launch &L, cudaGraphConditionalHandle cond, const int *flag, bool negate) {
  L.tick();
  k_flag_condition<<<1, 1, 0, L.stream>>>(cond, flag, negate ? 1 : 0);
}

}  // namespace pism_gpu
