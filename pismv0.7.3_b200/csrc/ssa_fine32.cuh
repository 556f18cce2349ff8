// ssa_fine32.cuh — the fine-level SSAFD operator in FP32 (the multigrid smoother and the
// inner solves of the mixed-precision path): FP32 copies of nu*H, beta and the inverse
// diagonal blocks, refreshed once per Picard iteration, and the stencil applied from
// shared-memory halo tiles.
#pragma once

#include "ssa_internal.h"
#include "ssa_stencil.cuh"

namespace pism_gpu {

__device__ __forceinline__ float4 inv2x2(float a11, float a12, float a21, float a22) {
  const float det = a11 * a22 - a12 * a21;
  if (det != 0.0f && isfinite(det)) {
    const float r = 1.0f / det;
    return make_float4(a22 * r, -a12 * r, -a21 * r, a11 * r);
  }
  return make_float4(a11 != 0.0f ? 1.0f / a11 : 0.0f, 0.0f, 0.0f, a22 != 0.0f ? 1.0f / a22 : 0.0f);
}

__device__ __forceinline__ float2 fmul4(const float4 &m, const float2 &v) {
  return make_float2(m.x * v.x + m.y * v.y, m.z * v.x + m.w * v.y);
}

// ---------------------------------------------------------------------------
// fine-level FP32 data (once per Picard iteration)
// ---------------------------------------------------------------------------
struct FineF {
  GridDev g;
  float rdx2, rdy2, r2, r4, scaling, nu_bedrock;
  const uint32_t *flags;
  const float2 *nuH;    // FP32 nu*H
  const float *beta;    // FP32 beta
  const float4 *dinv;   // FP32 inverse diagonal blocks
  const double *H;      // thickness, read only where F_NB_* flags are set
};


// rows / apply of a fine cell from staged tiles
// the two FP32 rows of fine cell (i, j) from a staged tile of FP32 nu*H; false for a
// diagonal-only row
__device__ __forceinline__ bool fine_rows_tile(const FineF &F, int i, int j, uint32_t f, float bta,
                                               const HaloTile<float2> &nT, int ti, int tj, Row2T<float> &e1,
                                               Row2T<float> &e2) {
  if (f & F_DIAG_ONLY) return false;
  const GridDev &g = F.g;
  float c_w = nT[ti][tj + 1].x, c_e = nT[ti + 1][tj + 1].x, c_s = nT[ti + 1][tj].y, c_n = nT[ti + 1][tj + 1].y;
  if (f & F_NB_ANY) {   // nu_bedrock_set overrides, SSAFD.cc:561-585
    const int k = cell(g, i, j);
    const double Hc = F.H[k], HE = F.H[nbr(g, i, j, 1, 0)];
    if (f & F_NB_W) c_w = (float)(F.nu_bedrock * 0.5 * (Hc + F.H[nbr(g, i, j, -1, 0)]));
    if (f & F_NB_E) c_e = (float)(F.nu_bedrock * 0.5 * (Hc + HE));
    if (f & F_NB_N) c_n = (float)(F.nu_bedrock * 0.5 * (Hc + F.H[nbr(g, i, j, 0, 1)]));
    if (f & F_NB_S) c_s = (float)(F.nu_bedrock * 0.5 * (Hc + HE));
  }
  stencil_rows_t<float>(F.rdx2, F.rdy2, F.r2, F.r4, f, c_w, c_e, c_s, c_n, bta, e1, e2);
  return true;
}

// y = A x at fine cell (i, j) from its flag word f, beta, the four staggered nu*H
// coefficients (west, east, south, north faces) and x read through xr(di, dj)
template <class XR>
__device__ __forceinline__ float2 fine_apply_coef(const FineF &F, int i, int j, uint32_t f, float bta, float c_w,
                                                  float c_e, float c_s, float c_n, const XR &xr) {
  if ((f & (F_WEIGHTS | F_DIAG_ONLY | F_NB_ANY)) == F_WEIGHTS)
    return apply_regular<float, float2>(F.rdx2, F.rdy2, F.r2, F.r4, c_w, c_e, c_s, c_n, bta, xr);
  if (f & F_DIAG_ONLY) {
    const float2 xc = xr(0, 0);
    return make_float2(F.scaling * xc.x, F.scaling * xc.y);
  }
  if (f & F_NB_ANY) {   // nu_bedrock_set overrides, SSAFD.cc:561-585
    const GridDev &g = F.g;
    const int k = cell(g, i, j);
    const double Hc = F.H[k], HE = F.H[nbr(g, i, j, 1, 0)];
    if (f & F_NB_W) c_w = (float)(F.nu_bedrock * 0.5 * (Hc + F.H[nbr(g, i, j, -1, 0)]));
    if (f & F_NB_E) c_e = (float)(F.nu_bedrock * 0.5 * (Hc + HE));
    if (f & F_NB_N) c_n = (float)(F.nu_bedrock * 0.5 * (Hc + F.H[nbr(g, i, j, 0, 1)]));
    if (f & F_NB_S) c_s = (float)(F.nu_bedrock * 0.5 * (Hc + HE));
  }
  Row2T<float> e1, e2;
  stencil_rows_t<float>(F.rdx2, F.rdy2, F.r2, F.r4, f, c_w, c_e, c_s, c_n, bta, e1, e2);
  return apply_rows_rel<float, float2>(e1, e2, xr);
}

// y = A x at fine cell (i, j) = tile position (ti, tj), x and nu*H from tiles
// f and bta (the cell's flag word and beta) are loaded by the caller together with the
// halo tiles, so that a tile costs one round trip to memory
__device__ __forceinline__ float2 fine_apply_tile(const FineF &F, int i, int j, uint32_t f, float bta,
                                                  const HaloTile<float2> &xT, const HaloTile<float2> &nT, int ti,
                                                  int tj) {
  auto xr = [&](int di, int dj) { return xT[ti + 1 + di][tj + 1 + dj]; };
  return fine_apply_coef(F, i, j, f, bta, nT[ti][tj + 1].x, nT[ti + 1][tj + 1].x, nT[ti + 1][tj].y,
                         nT[ti + 1][tj + 1].y, xr);
}


__device__ __forceinline__ float2 to_f2(const double2 &v) { return make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ float2 to_f2(const float2 &v) { return v; }
template <class V>
__device__ __forceinline__ V from_f2(const float2 &v);
template <>
__device__ __forceinline__ double2 from_f2<double2>(const float2 &v) { return make_double2((double)v.x, (double)v.y); }
template <>
__device__ __forceinline__ float2 from_f2<float2>(const float2 &v) { return v; }

FineF fine_view(const GridDev &g, const Fields &f, const MGHierarchy &H);

// right-hand side accessors of the fine-level multigrid passes: b(q) is the value at cell q.
// A kernel calls bind() once at its start (after the early exit of a finished solve).
template <class V>
struct VecAcc {   // a stored vector
  const V *p;
  __device__ __forceinline__ VecAcc bind() const { return *this; }
  __device__ __forceinline__ float2 operator()(int q) const { return to_f2(p[q]); }
};
// BiCGStab's s = r - alpha v, formed where it is read instead of stored (alpha from the
// device-side Krylov state, as the iteration's other kernels read it)
struct SAcc {
  const float2 *r, *v;
  const KState *st;
  float al;
  __device__ __forceinline__ SAcc bind() const { return SAcc{r, v, st, (float)st->alpha}; }
  __device__ __forceinline__ float2 operator()(int q) const {
    const float2 rk = r[q], vk = v[q];
    return make_float2(rk.x - al * vk.x, rk.y - al * vk.y);
  }
};

}  // namespace pism_gpu
