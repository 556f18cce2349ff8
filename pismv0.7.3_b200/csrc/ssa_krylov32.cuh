// ssa_krylov32.cuh — what the FP32 BiCGStab does with each operator apply y = A x: the two
// epilogues of the inner iteration, shared by the apply kernels of ssa_mixed.cu and by the
// multigrid fine-level pass fused with them (ssa_mg.cu), so both routes give the same bits.
//
//   EpiV:  v = A phat, alpha = rho / (rhat, v)
//   EpiT:  t = A shat, omega = (t, s) / (t, t), s = r - alpha v formed where it is read
//
// Each thread accumulates its cells' terms in FP64 in tile order; finish() adds the grid's
// partial sums in block order (ssa_reduce.cuh) and writes the scalar to the Krylov state.
#pragma once

#include "ssa_reduce.cuh"

namespace pism_gpu {

__device__ __forceinline__ double dotf(const float2 &a, const float2 &b) {
  return (double)a.x * (double)b.x + (double)a.y * (double)b.y;
}

struct EpiV {
  const float2 *rhat;
  float2 *v;
  double *partials;
  unsigned *ticket;
  KState *st;
  double acc[1];

  __device__ __forceinline__ void begin() { acc[0] = 0.0; }
  __device__ __forceinline__ void body(int k, const float2 &y) {
    v[k] = y;
    acc[0] += dotf(rhat[k], y);
  }
  __device__ __forceinline__ void finish() {
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
};

struct EpiT {
  const float2 *r, *v;
  float2 *t;
  double *partials;
  unsigned *ticket;
  KState *st;
  double acc[2];
  float al;

  __device__ __forceinline__ void begin() {
    acc[0] = acc[1] = 0.0;
    al = (float)st->alpha;
  }
  __device__ __forceinline__ void body(int k, const float2 &y) {
    t[k] = y;
    const float2 rk = r[k], vk = v[k];
    acc[0] += dotf(y, make_float2(rk.x - al * vk.x, rk.y - al * vk.y));
    acc[1] += dotf(y, y);
  }
  __device__ __forceinline__ void finish() {
    double tot[2];
    if (grid_reduce<2>(acc, partials, ticket, tot)) st->omega = (tot[1] != 0.0) ? tot[0] / tot[1] : 0.0;
  }
};

}  // namespace pism_gpu
