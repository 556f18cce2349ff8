// ssa_reduce.cuh — grid-wide sums fused into a producing kernel: each block writes its
// partial sums, the last block to finish (atomic ticket) adds them in block order (so
// the result is deterministic) and may update solver scalars on the device.
#pragma once

#include "ssa_internal.h"

namespace pism_gpu {

constexpr int RED_THREADS = 256;   // every reducing kernel runs 256-thread blocks

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Reduce NV values over the grid.  Returns true in thread 0 of the last block,
// with the grid totals in tot[].
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&val)[NV], double *partials, unsigned *ticket,
                                            double (&tot)[NV]) {
  __shared__ double sh[NV][RED_THREADS / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double s = warp_sum(val[v]);
    if (lane == 0) sh[v][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = 0.0;
      for (int w = 0; w < RED_THREADS / 32; ++w) s += sh[v][w];
      partials[blockIdx.x * NV + v] = s;
    }
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // the last block adds all partials in block order (deterministic)
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += RED_THREADS) s += __ldcg(&partials[b * NV + v]);
    s = warp_sum(s);
    if (lane == 0) sh[v][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x != 0) return false;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double s = 0.0;
    for (int w = 0; w < RED_THREADS / 32; ++w) s += sh[v][w];
    tot[v] = s;
  }
  *ticket = 0u;
  return true;
}

}  // namespace pism_gpu
