// ssa_control.cu — device-side control of the Picard loop.
//
// A whole SSAFD solve (SSAFD::picard_manager, SSAFD.cc:962-1119, with its linear solves) can
// run as one CUDA graph whose conditional WHILE / IF nodes take their values from a PState
// in device memory.  These single-thread kernels make the decisions the host loop makes, in
// the same double arithmetic, so the graph takes the same path: the KSP tolerance of each
// Picard iteration (inexact Picard), the refinement steps of the mixed-precision solve, the
// zero-diagonal and KSP-failure checks and the Picard stopping test (SSAFD.cc:1084).  The
// decisions themselves are the __host__ __device__ functions of ssa_state.h; these kernels
// apply them to the state in device memory.
#include <climits>

#include "ssa_internal.h"

namespace pism_gpu {
namespace {

__global__ void k_picard_start(PState *P) { picard_start(*P); }

__global__ void k_picard_begin(PState *P, PicardConst c, int *zero_diag_cell) {
  *zero_diag_cell = INT_MAX;
  picard_begin(*P, c);
}

__global__ void k_ksp_begin(KState *st, const PState *P, int maxit) { ksp_begin(*st, *P, maxit); }

__global__ void k_ksp_end(PState *P, const KState *st, int body_iters) { ksp_end(*P, *st, body_iters); }

__global__ void k_refine_end(PState *P, const KState *st, int max_refine) { refine_end(*P, *st, max_refine); }

__global__ void k_picard_after_solve(PState *P, const int *zero_diag_cell) {
  picard_after_solve(*P, *zero_diag_cell);
}

__global__ void k_picard_test(PState *P, const double *norm2, PicardConst c) {
  picard_test(*P, norm2[0], norm2[1], c);
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
