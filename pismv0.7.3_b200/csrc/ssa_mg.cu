// ssa_mg.cu — aggregation multigrid preconditioner for the SSAFD system (replaces the
// reference's PETSc block-Jacobi / ILU(0) and ASM / LU preconditioners,
// SSAFD.cc:136-219, inside the Krylov solve).  It runs in FP32: it only has to
// approximate A^-1; the Krylov method around it, the operator and the residuals stay FP64.
//
// Hierarchy: level 0 is the fine SSAFD operator, applied matrix-free from an FP32 copy of
// nu*H and beta (refreshed once per Picard iteration) and the flag word.  Level l+1
// aggregates 2 x 2 cells of level l (1 in a direction that is already <= 4 cells) and
// carries the Galerkin operator R A P with piecewise-constant P (R = P^T): the sum, over
// the aggregate, of the fine 2 x 2 blocks grouped by the neighbouring aggregate they
// couple to.  With a 3 x 3 fine stencil this is again a 3 x 3 stencil of 2 x 2 blocks,
// stored as 9 float4 arrays (one per block) so that a warp reads 512 contiguous bytes per
// block.  The coarsest level (<= 4 x 4 cells) is inverted densely in FP64.
//
// Cycle (a V(1,1) cycle used as a fixed preconditioner z = M^-1 b):
//   x_l = omega D_l^-1 b_l                       (computed on the fly, never stored)
//   b_{l+1} = R (b_l - A_l x_l)                  (restriction kernel)
//   ...  x_L = A_L^-1 b_L                        (dense inverse)
//   x_l <- x_l + s P x_{l+1};  x_l <- x_l + omega D_l^-1 (b_l - A_l x_l)   (post kernel)
// so each level costs two stencil passes.  Levels of <= MG_CTA_CELLS cells are cycled by
// one thread-block cluster in one launch (their kernels would be launch- and
// latency-bound), and their Galerkin operators and the coarsest inverse are built by one
// cluster launch per Picard iteration.
// The defaults omega = 0.9 and s = 1.2 (mg_omega, mg_correction; s > 1 over-corrects to
// compensate the piecewise-constant interpolation) come from a sweep of whole 801^2
// synthetic solves: 7115 BiCGStab iterations against 9558 at (0.7, 1.5) and 8042 at
// (0.85, 1.5); omega >= 1 makes the damped block-Jacobi smoother unstable (> 1e5).
#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include <cooperative_groups.h>

#include "ssa_fine32.cuh"
#include "ssa_krylov32.cuh"
#include "ssa_small_plan.h"

namespace pism_gpu {
namespace cg = cooperative_groups;

namespace {

constexpr int TJm = 32, TIm = 8, NTm = TJm * TIm;
constexpr int CTA_THREADS = 1024;
constexpr int SMALL_CLUSTER = 8;   // CTAs (SMs) of the cluster that cycles the small levels
static_assert(SMALL_CLUSTER == SC_CTAS, "the shared-memory cycle's split assumes the cluster size");
// dynamic shared memory of the shared-memory cycle (the kernel's static part is < 2 KB)
constexpr int SMALL_DSMEM_MAX_BYTES = 220 * 1024;

struct TileM {
  int tiles_j, tiles;
};

TileM tiles_of(int Mx, int My) {
  TileM t;
  t.tiles_j = (My + TJm - 1) / TJm;
  t.tiles = t.tiles_j * ((Mx + TIm - 1) / TIm);
  return t;
}

__device__ __forceinline__ bool tile_cell(const TileM &tm, int Mx, int My, int t, int &i, int &j) {
  const int ti = t / tm.tiles_j, tj = t - ti * tm.tiles_j;
  j = tj * TJm + (threadIdx.x & (TJm - 1));
  i = ti * TIm + (threadIdx.x >> 5);
  return i < Mx && j < My;
}

__device__ __forceinline__ int wdiff(int a, int b, int n) {
  int d = a - b;
  if (d > 1) d -= n;
  if (d < -1) d += n;
  return d;
}

// stencil block index of the offset (di, dj): NW N NE / W C E / SW S SE
__host__ __device__ __forceinline__ int blk_of(int di, int dj) { return (1 - dj) * 3 + (di + 1); }

struct LevelView {
  int Mx, My, N, ax, ay;
  const float4 *A;     // 9 blocks x N: block b of cell k at A[b * N + k]
  const float4 *dinv;
  float2 *b, *x;
};

// y = A_l x at (i, j), x read through xa(i', j')
template <class XA>
__device__ __forceinline__ float2 coarse_apply(const LevelView &L, int i, int j, const XA &xa) {
  const int k = i * L.My + j;
  const int ip = wrap(i + 1, L.Mx), im = wrap(i - 1, L.Mx), jp = wrap(j + 1, L.My), jm = wrap(j - 1, L.My);
  const int ii[9] = {im, i, ip, im, i, ip, im, i, ip};
  const int jj[9] = {jp, jp, jp, j, j, j, jm, jm, jm};
  float4 a[9];
#pragma unroll
  for (int b = 0; b < 9; ++b) a[b] = L.A[b * L.N + k];
  float y1 = 0.0f, y2 = 0.0f;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const float2 xv = xa(ii[b], jj[b]);
    y1 += a[b].x * xv.x + a[b].y * xv.y;
    y2 += a[b].z * xv.x + a[b].w * xv.y;
  }
  return make_float2(y1, y2);
}

// FP32 copies of nu*H, beta and D^-1 for the fine-level passes (once per Picard iteration)
__global__ void k_mg0_compact(int N, const double2 *__restrict__ nuH, const double *__restrict__ beta,
                              const double4 *__restrict__ dinv, float2 *__restrict__ nuHf, float *__restrict__ betaf,
                              float4 *__restrict__ dinvf) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double2 n = nuH[k];
    const double4 d = dinv[k];
    nuHf[k] = make_float2((float)n.x, (float)n.y);
    betaf[k] = (float)beta[k];
    dinvf[k] = make_float4((float)d.x, (float)d.y, (float)d.z, (float)d.w);
  }
}

// ---------------------------------------------------------------------------
// set-up: Galerkin coarse operators
// ---------------------------------------------------------------------------
// acc[4 cb .. 4 cb + 3] += (x, y, z, w) for a block index cb known only at run time: the
// accumulators stay in registers (every index below is static once unrolled), so the
// operator loads of the next fine cell need not wait behind shared-memory updates
__device__ __forceinline__ void acc_block(double (&acc)[36], int cb, double x, double y, double z, double w) {
#pragma unroll
  for (int c = 0; c < 9; ++c)
    if (cb == c) {
      acc[4 * c + 0] += x;
      acc[4 * c + 1] += y;
      acc[4 * c + 2] += z;
      acc[4 * c + 3] += w;
    }
}

// the coarse cell's nine blocks (FP32) and its D^-1 from the FP64 sums
__device__ __forceinline__ void store_coarse(const double (&acc)[36], int Nc, int kc, float4 *Ac, float4 *dinvc) {
#pragma unroll
  for (int b = 0; b < 9; ++b)
    Ac[b * Nc + kc] = make_float4((float)acc[4 * b], (float)acc[4 * b + 1], (float)acc[4 * b + 2], (float)acc[4 * b + 3]);
  dinvc[kc] = inv2x2((float)acc[16], (float)acc[17], (float)acc[18], (float)acc[19]);
}

// Whether the coarse blocks of a fine cell's nine blocks follow from its place in a 2 x 2
// aggregate alone: floor((p + d) / 2) for fine offset p in {0, 1} and stencil offset d.
// That holds for 2 x 2 aggregation with >= 3 coarse cells each way (the periodic wrap then
// only links the first and last aggregates, at offset -1 / +1 as in the interior), except
// that on a level with an odd number of cells the last aggregate is one cell wide and its
// wrapped east (north) neighbour is the first aggregate, one further (ex, ey).
__device__ __forceinline__ bool static_blocks(int ax, int ay, int Mxc, int Myc) {
  return ax == 2 && ay == 2 && Mxc >= 3 && Myc >= 3;
}

// acc += the nine blocks v(b) of fine cell (PI, PJ) of its aggregate, each to its coarse
// block (static_blocks); the additions in block order, as acc_block would make them
template <int PI, int PJ, class V>
__device__ __forceinline__ void acc_fine_static(double (&acc)[36], bool ex, bool ey, const V &v) {
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const int di = (b % 3) - 1, dj = 1 - (b / 3);
    const int ci = (PI + di + 2) / 2 - 1, cj = (PJ + dj + 2) / 2 - 1;   // floor((p + d) / 2)
    const bool wx = PI == 0 && di == 1, wy = PJ == 0 && dj == 1;       // may cross the odd edge
    const double4 x = v(b);
    if (wx || wy) {
      acc_block(acc, blk_of(ci + (wx && ex ? 1 : 0), cj + (wy && ey ? 1 : 0)), x.x, x.y, x.z, x.w);
    } else {
      const int cb = blk_of(ci, cj);
      acc[4 * cb + 0] += x.x;
      acc[4 * cb + 1] += x.y;
      acc[4 * cb + 2] += x.z;
      acc[4 * cb + 3] += x.w;
    }
  }
}

// level 1 from the fine operator (FP64 rows, FP64 accumulation in registers)
__global__ void __launch_bounds__(NTm) k_mg_build1(GridDev g, StencilConst s, const uint32_t *__restrict__ flags,
                                                   const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                                   int ax, int ay, int Mxc, int Myc, TileM tm, float4 *Ac,
                                                   float4 *dinvc) {
  const int Nc = Mxc * Myc;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int I, J;
    if (!tile_cell(tm, Mxc, Myc, t, I, J)) continue;
    double acc[36];
#pragma unroll
    for (int q = 0; q < 36; ++q) acc[q] = 0.0;
    const bool fast = static_blocks(ax, ay, Mxc, Myc);
    const bool ex = (g.Mx & 1) && I == Mxc - 1, ey = (g.My & 1) && J == Myc - 1;
    // the two rows of fine cell (pi, pj), added to its coarse blocks
    auto fine = [&](auto PI, auto PJ) {
      const int pi = decltype(PI)::value, pj = decltype(PJ)::value;
      const int i = I * ax + pi, j = J * ay + pj;
      if (pi >= ax || pj >= ay || i >= g.Mx || j >= g.My) return;
      const uint32_t f = flags[cell(g, i, j)];
      Row2 e1, e2;
      if (!cell_rows(g, s, i, j, f, nuH, beta, e1, e2)) {
        acc[4 * blk_of(0, 0) + 0] += s.scaling;
        acc[4 * blk_of(0, 0) + 3] += s.scaling;
        return;
      }
      const double r1u[9] = {e1.uNW, e1.uN, e1.uNE, e1.uW, e1.uC, e1.uE, e1.uSW, e1.uS, e1.uSE};
      const double r1v[9] = {e1.vNW, e1.vN, e1.vNE, e1.vW, e1.vC, e1.vE, e1.vSW, e1.vS, e1.vSE};
      const double r2u[9] = {e2.uNW, e2.uN, e2.uNE, e2.uW, e2.uC, e2.uE, e2.uSW, e2.uS, e2.uSE};
      const double r2v[9] = {e2.vNW, e2.vN, e2.vNE, e2.vW, e2.vC, e2.vE, e2.vSW, e2.vS, e2.vSE};
      auto v = [&](int b) { return make_double4(r1u[b], r1v[b], r2u[b], r2v[b]); };
      if (fast) {
        acc_fine_static<decltype(PI)::value, decltype(PJ)::value>(acc, ex, ey, v);
      } else {
#pragma unroll
        for (int b = 0; b < 9; ++b) {
          const int di = (b % 3) - 1, dj = 1 - (b / 3);
          const int ni = wrap(i + di, g.Mx), nj = wrap(j + dj, g.My);
          acc_block(acc, blk_of(wdiff(ni / ax, I, Mxc), wdiff(nj / ay, J, Myc)), r1u[b], r1v[b], r2u[b], r2v[b]);
        }
      }
    };
    fine(std::integral_constant<int, 0>{}, std::integral_constant<int, 0>{});
    fine(std::integral_constant<int, 0>{}, std::integral_constant<int, 1>{});
    fine(std::integral_constant<int, 1>{}, std::integral_constant<int, 0>{});
    fine(std::integral_constant<int, 1>{}, std::integral_constant<int, 1>{});
    store_coarse(acc, Nc, I * Myc + J, Ac, dinvc);
  }
}

// Galerkin operator and D^-1 of coarse cell (I, J) of the level below F, summed in FP64 in
// registers, fine cell by fine cell of the aggregate and block by block (no stores between
// the loads, so the compiler may issue them all at once)
__device__ __forceinline__ void galerkin_cell(const LevelView &F, int Mxc, int Myc, int I, int J, float4 *Ac,
                                              float4 *dinvc) {
  const int ax = F.ax, ay = F.ay;
  double acc[36];
#pragma unroll
  for (int q = 0; q < 36; ++q) acc[q] = 0.0;
  const bool fast = static_blocks(ax, ay, Mxc, Myc);
  const bool ex = (F.Mx & 1) && I == Mxc - 1, ey = (F.My & 1) && J == Myc - 1;
  auto fine = [&](auto PI, auto PJ) {
    constexpr int pi = decltype(PI)::value, pj = decltype(PJ)::value;
    const int i = I * ax + pi, j = J * ay + pj;
    if (pi >= ax || pj >= ay || i >= F.Mx || j >= F.My) return;
    const int k = i * F.My + j;
    auto v = [&](int b) {
      const float4 a = F.A[b * F.N + k];
      return make_double4(a.x, a.y, a.z, a.w);
    };
    if (fast) {
      acc_fine_static<pi, pj>(acc, ex, ey, v);
    } else {
#pragma unroll
      for (int b = 0; b < 9; ++b) {
        const int di = (b % 3) - 1, dj = 1 - (b / 3);
        const int ni = wrap(i + di, F.Mx), nj = wrap(j + dj, F.My);
        const double4 x = v(b);
        acc_block(acc, blk_of(wdiff(ni / ax, I, Mxc), wdiff(nj / ay, J, Myc)), x.x, x.y, x.z, x.w);
      }
    }
  };
  fine(std::integral_constant<int, 0>{}, std::integral_constant<int, 0>{});
  fine(std::integral_constant<int, 0>{}, std::integral_constant<int, 1>{});
  fine(std::integral_constant<int, 1>{}, std::integral_constant<int, 0>{});
  fine(std::integral_constant<int, 1>{}, std::integral_constant<int, 1>{});
  store_coarse(acc, Mxc * Myc, I * Myc + J, Ac, dinvc);
}

// level l+1 from the stored operator of level l
__global__ void __launch_bounds__(NTm, 2) k_mg_build(LevelView F, int Mxc, int Myc, TileM tm, float4 *Ac, float4 *dinvc) {
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    int I, J;
    if (!tile_cell(tm, Mxc, Myc, t, I, J)) continue;
    galerkin_cell(F, Mxc, Myc, I, J, Ac, dinvc);
  }
}

// Dense inverse of the coarsest operator (n = 2 N <= 32 unknowns) by Gauss-Jordan elimination
// with partial pivoting, in place in shared memory, by one thread block (rows padded to 33
// entries, so a column's entries of consecutive rows sit in different banks).  Warp 0 finds
// each pivot, swaps and scales the pivot row (two block barriers per step in all); the
// elimination spreads the n x n element updates of a step over the block,
// reading the step's multipliers from a copy of the pivot column, so each element is updated
// with the same operands in the same order whatever thread does it.  Written transposed, so
// that the per-cycle product reads it coalesced.
constexpr int CI_PAD = 2 * MG_MAX_COARSE_CELLS + 1;
static_assert(2 * MG_MAX_COARSE_CELLS <= 32, "one lane per row of the coarsest operator");

struct CoarseInvertSmem {
  double a[2 * MG_MAX_COARSE_CELLS][CI_PAD];
  double fcol[2 * MG_MAX_COARSE_CELLS];
  int perm[2 * MG_MAX_COARSE_CELLS];
};

__device__ void coarse_invert_block(const LevelView &L, CoarseInvertSmem &S, double *invT_out, int *singular) {
  const int tid = threadIdx.x, nth = blockDim.x, n = 2 * L.N;
  for (int q = tid; q < n * CI_PAD; q += nth) (&S.a[0][0])[q] = 0.0;
  __syncthreads();
  if (tid < L.N) {   // each cell's two rows are written by one thread
    const int k = tid, i = k / L.My, j = k % L.My;
    for (int b = 0; b < 9; ++b) {
      const int di = (b % 3) - 1, dj = 1 - (b / 3);
      const int kn = wrap(i + di, L.Mx) * L.My + wrap(j + dj, L.My);
      const float4 v = L.A[b * L.N + k];
      S.a[2 * k + 0][2 * kn + 0] += (double)v.x;
      S.a[2 * k + 0][2 * kn + 1] += (double)v.y;
      S.a[2 * k + 1][2 * kn + 0] += (double)v.z;
      S.a[2 * k + 1][2 * kn + 1] += (double)v.w;
    }
  }
  __syncthreads();
  for (int col = 0; col < n; ++col) {
    // warp 0: the pivot (the largest |a[r][col]|, r >= col, lowest row on ties), the row
    // interchange, the scaled pivot row and the copy of the multipliers, ordered by __syncwarp
    if (tid < 32) {
      const int t = tid;
      double best = -1.0;
      int bi = col;
      if (col + t < n) {
        best = fabs(S.a[col + t][col]);
        bi = col + t;
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (t == 0) {
        S.perm[col] = bi;
        if (!(best > 0.0)) *singular = 1;
      }
      const int p = bi;
      if (p != col && t < n) {   // lane t swaps column t of the two rows
        const double tmp = S.a[col][t];
        S.a[col][t] = S.a[p][t];
        S.a[p][t] = tmp;
      }
      __syncwarp();
      const double pv = S.a[col][col];
      const double pinv = pv != 0.0 ? 1.0 / pv : 0.0;
      __syncwarp();
      // pivot row: a[col][col] <- 1, then scaled by 1 / pivot (so it holds 1 / pivot); the
      // multipliers of the other rows are copied before any of them changes
      if (t < n) {
        S.a[col][t] = (t == col ? 1.0 : S.a[col][t]) * pinv;
        S.fcol[t] = S.a[t][col];
      }
    }
    __syncthreads();
    // other rows: a[r][q] -= a[r][col] a[col][q]; a[r][col] <- -a[r][col] / pivot (element e
    // is (r, q) = (e / 32, e % 32), those outside n x n idle)
    for (int e = tid; e < 32 * 32; e += nth) {
      const int r = e >> 5, q = e & 31;
      if (r == col || r >= n || q >= n) continue;
      const double f = S.fcol[r];
      if (q != col) S.a[r][q] -= f * S.a[col][q];
      else S.a[r][col] = -f * S.a[col][col];
    }
    __syncthreads();
  }
  // undo the row interchanges as column interchanges, in reverse order
  for (int col = n - 1; col >= 0; --col) {
    const int p = S.perm[col];
    if (p != col && tid < n) {
      const double tmp = S.a[tid][col];
      S.a[tid][col] = S.a[tid][p];
      S.a[tid][p] = tmp;
    }
    __syncthreads();
  }
  for (int q = tid; q < n * n; q += nth) {
    const int c = q / n, r = q - c * n;
    invT_out[q] = S.a[r][c];   // invT[c][r] = inverse[r][c]
  }
}

// the coarsest inverse, after the last level build (CI_THREADS threads: one element of the
// 32 x 32 elimination each)
constexpr int CI_THREADS = 1024;
__global__ void __launch_bounds__(CI_THREADS) k_mg_coarse_invert(LevelView L, double *invT_out, int *singular) {
  __shared__ CoarseInvertSmem S;
  coarse_invert_block(L, S, invT_out, singular);
}

// The small levels' Galerkin operators (levels first .. nlev - 1, each from the level above it,
// all of <= MG_CTA_CELLS cells) and the coarsest inverse in one launch on one thread-block
// cluster: one cluster barrier (release / acquire at cluster scope) between levels; the
// coarsest inverse follows as its own launch.  The arithmetic of every cell is k_mg_build's.
__global__ void __cluster_dims__(SMALL_CLUSTER, 1, 1) __launch_bounds__(NTm)
    k_mg_build_small(const LevelView *__restrict__ lev, int first, int nlev) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = cluster.block_rank() * NTm + threadIdx.x, nthr = SMALL_CLUSTER * NTm;
  for (int c = first; c < nlev; ++c) {
    const LevelView F = lev[c - 1], C = lev[c];
    for (int kc = rank; kc < C.N; kc += nthr) {
      const int I = kc / C.My, J = kc - I * C.My;
      galerkin_cell(F, C.Mx, C.My, I, J, const_cast<float4 *>(C.A), const_cast<float4 *>(C.dinv));
    }
    cluster.sync();
  }
}

// ---------------------------------------------------------------------------
// V-cycle kernels
// ---------------------------------------------------------------------------
// y = A_l x at coarse cell = tile position (ti, tj); a[] = the cell's 9 stencil blocks,
// loaded by the caller together with the tile
__device__ __forceinline__ float2 coarse_apply_tile(const float4 (&a)[9], const HaloTile<float2> &xT, int ti, int tj) {
  float y1 = 0.0f, y2 = 0.0f;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const int di = (b % 3) - 1, dj = 1 - (b / 3);
    const float2 xv = xT[ti + 1 + di][tj + 1 + dj];
    y1 += a[b].x * xv.x + a[b].y * xv.y;
    y2 += a[b].z * xv.x + a[b].w * xv.y;
  }
  return make_float2(y1, y2);
}

// 2 x 2 (AX x AY) aggregate sums of the residuals staged in rsh, written to bc
template <int AX, int AY>
__device__ __forceinline__ void store_aggregates(float2 (&rsh)[TILE_I][TILE_J], int i0, int j0, int Mxc, int Myc,
                                                 float2 *__restrict__ bc) {
  constexpr int CJ = TILE_J / AY, CI = TILE_I / AX;
  if (threadIdx.x < CI * CJ) {
    const int ci = threadIdx.x / CJ, cj = threadIdx.x - ci * CJ;
    float ru = 0.0f, rv = 0.0f;
#pragma unroll
    for (int pi = 0; pi < AX; ++pi)
#pragma unroll
      for (int pj = 0; pj < AY; ++pj) {
        const float2 r = rsh[ci * AX + pi][cj * AY + pj];
        ru += r.x;
        rv += r.y;
      }
    const int I = i0 / AX + ci, J = j0 / AY + cj;
    if (I < Mxc && J < Myc) bc[I * Myc + J] = make_float2(ru, rv);
  }
}

// fine level: b_1 = R (b - A x0), x0 = omega D^-1 b
template <int AX, int AY, class BA>
__global__ void __launch_bounds__(NTm) k_mg0_restrict(FineF F, BA b_in, float omega, int Mxc,
                                                      int Myc, TileM tm, float2 *__restrict__ bc, const KState *st) {
  if (st && st->done) return;
  const auto b = b_in.bind();
  __shared__ HaloTile<float2> xT, nT;
  __shared__ float2 rsh[TILE_I][TILE_J];
  const GridDev &g = F.g;
  const int ti = threadIdx.x >> 5, tj = threadIdx.x & 31;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    const int i0 = (t / tm.tiles_j) * TILE_I, j0 = (t % tm.tiles_j) * TILE_J;
    const int i = i0 + ti, j = j0 + tj;
    const bool inside = i < g.Mx && j < g.My;
    const int k = inside ? i * g.My + j : 0;
    const uint32_t f = F.flags[k];   // issued with the tile loads: one round trip per tile
    const float bta = F.beta[k];
    const float2 bk = b(k);
    __syncthreads();
    load_halo_tile<float2>(xT, i0, j0, g.Mx, g.My, [&](int ii, int jj) {
      const int q = ii * g.My + jj;
      const float2 v = fmul4(F.dinv[q], b(q));
      return make_float2(omega * v.x, omega * v.y);
    });
    load_halo_tile<float2>(nT, i0, j0, g.Mx, g.My, [&](int ii, int jj) { return F.nuH[ii * g.My + jj]; });
    __syncthreads();
    float2 r = make_float2(0.0f, 0.0f);
    if (inside) {
      const float2 y = fine_apply_tile(F, i, j, f, bta, xT, nT, ti, tj);
      r = make_float2(bk.x - y.x, bk.y - y.y);
    }
    rsh[ti][tj] = r;
    __syncthreads();
    store_aggregates<AX, AY>(rsh, i0, j0, Mxc, Myc, bc);
  }
}

// fine level: x = omega D^-1 b + s P x_1;  z = x + omega D^-1 (b - A x)
template <int AX, int AY, class BA, class ZV>
__global__ void __launch_bounds__(NTm) k_mg0_post(FineF F, BA b_in, float omega, float corr,
                                                  int Myc, const float2 *__restrict__ xc, TileM tm,
                                                  ZV *__restrict__ z, const KState *st) {
  if (st && st->done) return;
  const auto b = b_in.bind();
  __shared__ HaloTile<float2> xT, nT;
  const GridDev &g = F.g;
  const int ti = threadIdx.x >> 5, tj = threadIdx.x & 31;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    const int i0 = (t / tm.tiles_j) * TILE_I, j0 = (t % tm.tiles_j) * TILE_J;
    const int i = i0 + ti, j = j0 + tj;
    const bool inside = i < g.Mx && j < g.My;
    const int k = inside ? i * g.My + j : 0;
    const uint32_t f = F.flags[k];   // issued with the tile loads: one round trip per tile
    const float bta = F.beta[k];
    const float2 bk = b(k);
    const float4 dk = F.dinv[k];
    __syncthreads();
    load_halo_tile<float2>(xT, i0, j0, g.Mx, g.My, [&](int ii, int jj) {
      const int q = ii * g.My + jj;
      const float2 v = fmul4(F.dinv[q], b(q));
      const float2 c = xc[(ii / AX) * Myc + jj / AY];
      return make_float2(omega * v.x + corr * c.x, omega * v.y + corr * c.y);
    });
    load_halo_tile<float2>(nT, i0, j0, g.Mx, g.My, [&](int ii, int jj) { return F.nuH[ii * g.My + jj]; });
    __syncthreads();
    if (inside) {
      const float2 xk = xT[ti + 1][tj + 1];
      const float2 y = fine_apply_tile(F, i, j, f, bta, xT, nT, ti, tj);
      const float2 d = fmul4(dk, make_float2(bk.x - y.x, bk.y - y.y));
      z[k] = from_f2<ZV>(make_float2(xk.x + omega * d.x, xk.y + omega * d.y));
    }
  }
}

// The fine-level pass fused with the FP32 operator apply that follows the V-cycle in
// BiCGStab.  Per tile: x = omega D^-1 b + corr P x_1 on the tile and a two-cell halo;
// z = x + omega D^-1 (b - A x) on the tile and a one-cell halo (the halo's z recomputed here
// rather than read back from the tiles that own it); z stored on the tile; y = A z on the
// tile handed to the epilogue.  Every value comes from the same arithmetic as k_mg0_post
// followed by the apply kernel, over the same tiles in the same order per block, so the
// results and the epilogue's sums are the same bits.
constexpr int H2I = TIm + 4, H2J = TJm + 4;   // the two-cell-halo region of a tile

template <int AX, int AY, class BA, class EPI>
__global__ void __launch_bounds__(NTm) k_mg0_post_apply(FineF F, BA b_in, float omega, float corr, int Myc,
                                                        const float2 *__restrict__ xc, TileM tm,
                                                        float2 *__restrict__ z, EPI e) {
  if (e.st->done) return;
  e.begin();
  const auto b = b_in.bind();
  __shared__ float2 xs[H2I][H2J], ns[H2I][H2J], zs[TIm + 2][TJm + 2];
  const int Mx = F.g.Mx, My = F.g.My;
  const int ti = threadIdx.x >> 5, tj = threadIdx.x & 31;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    const int i0 = (t / tm.tiles_j) * TIm, j0 = (t % tm.tiles_j) * TJm;
    __syncthreads();   // the previous tile's readers are done
    for (int q = threadIdx.x; q < H2I * H2J; q += NTm) {   // cell (i0 - 2 + a, j0 - 2 + c), wrapped
      const int a = q / H2J, c = q - a * H2J;
      const int ii = pmod(i0 - 2 + a, Mx), jj = pmod(j0 - 2 + c, My), kq = ii * My + jj;
      const float2 v = fmul4(F.dinv[kq], b(kq));
      const float2 cc = xc[(ii / AX) * Myc + jj / AY];
      xs[a][c] = make_float2(omega * v.x + corr * cc.x, omega * v.y + corr * cc.y);
      ns[a][c] = F.nuH[kq];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (TIm + 2) * (TJm + 2); q += NTm) {   // cell (i0 - 1 + a, j0 - 1 + c)
      const int a = q / (TJm + 2), c = q - a * (TJm + 2);
      const int ii = pmod(i0 - 1 + a, Mx), jj = pmod(j0 - 1 + c, My), kq = ii * My + jj;
      auto xr = [&](int di, int dj) { return xs[a + 1 + di][c + 1 + dj]; };
      const float2 y = fine_apply_coef(F, ii, jj, F.flags[kq], F.beta[kq], ns[a][c + 1].x, ns[a + 1][c + 1].x,
                                       ns[a + 1][c].y, ns[a + 1][c + 1].y, xr);
      const float2 xk = xs[a + 1][c + 1], bk = b(kq);
      const float2 d = fmul4(F.dinv[kq], make_float2(bk.x - y.x, bk.y - y.y));
      zs[a][c] = make_float2(xk.x + omega * d.x, xk.y + omega * d.y);
    }
    __syncthreads();
    const int i = i0 + ti, j = j0 + tj;
    if (i < Mx && j < My) {
      const int k = i * My + j;
      z[k] = zs[ti + 1][tj + 1];
      auto zr = [&](int di, int dj) { return zs[ti + 1 + di][tj + 1 + dj]; };
      const float2 y = fine_apply_coef(F, i, j, F.flags[k], F.beta[k], ns[ti + 1][tj + 2].x, ns[ti + 2][tj + 2].x,
                                       ns[ti + 2][tj + 1].y, ns[ti + 2][tj + 2].y, zr);
      e.body(k, y);
    }
  }
  e.finish();
}

// coarse level l: b_{l+1} = R (b_l - A_l x0), x0 = omega D^-1 b_l
template <int AX, int AY>
__global__ void __launch_bounds__(NTm) k_mgc_restrict(LevelView L, float omega, int Mxc, int Myc, TileM tm,
                                                      float2 *__restrict__ bc, const KState *st) {
  if (st && st->done) return;
  __shared__ HaloTile<float2> xT;
  __shared__ float2 rsh[TILE_I][TILE_J];
  const int ti = threadIdx.x >> 5, tj = threadIdx.x & 31;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    const int i0 = (t / tm.tiles_j) * TILE_I, j0 = (t % tm.tiles_j) * TILE_J;
    const int i = i0 + ti, j = j0 + tj;
    const bool inside = i < L.Mx && j < L.My;
    const int k = inside ? i * L.My + j : 0;
    float4 a[9];   // issued with the tile loads: one round trip per tile
#pragma unroll
    for (int q = 0; q < 9; ++q) a[q] = L.A[q * L.N + k];
    const float2 bk = L.b[k];
    __syncthreads();
    load_halo_tile<float2>(xT, i0, j0, L.Mx, L.My, [&](int ii, int jj) {
      const int q = ii * L.My + jj;
      const float2 v = fmul4(L.dinv[q], L.b[q]);
      return make_float2(omega * v.x, omega * v.y);
    });
    __syncthreads();
    float2 r = make_float2(0.0f, 0.0f);
    if (inside) {
      const float2 y = coarse_apply_tile(a, xT, ti, tj);
      r = make_float2(bk.x - y.x, bk.y - y.y);
    }
    rsh[ti][tj] = r;
    __syncthreads();
    store_aggregates<AX, AY>(rsh, i0, j0, Mxc, Myc, bc);
  }
}

// coarse level l: x = omega D^-1 b + s P x_{l+1};  x <- x + omega D^-1 (b - A x)
template <int AX, int AY>
__global__ void __launch_bounds__(NTm) k_mgc_post(LevelView L, float omega, float corr, int Myc,
                                                  const float2 *__restrict__ xc, TileM tm, const KState *st) {
  if (st && st->done) return;
  __shared__ HaloTile<float2> xT;
  const int ti = threadIdx.x >> 5, tj = threadIdx.x & 31;
  for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
    const int i0 = (t / tm.tiles_j) * TILE_I, j0 = (t % tm.tiles_j) * TILE_J;
    const int i = i0 + ti, j = j0 + tj;
    const bool inside = i < L.Mx && j < L.My;
    const int k = inside ? i * L.My + j : 0;
    float4 a[9];   // issued with the tile loads: one round trip per tile
#pragma unroll
    for (int q = 0; q < 9; ++q) a[q] = L.A[q * L.N + k];
    const float2 bk = L.b[k];
    const float4 dk = L.dinv[k];
    __syncthreads();
    load_halo_tile<float2>(xT, i0, j0, L.Mx, L.My, [&](int ii, int jj) {
      const int q = ii * L.My + jj;
      const float2 v = fmul4(L.dinv[q], L.b[q]);
      const float2 c = xc[(ii / AX) * Myc + jj / AY];
      return make_float2(omega * v.x + corr * c.x, omega * v.y + corr * c.y);
    });
    __syncthreads();
    if (inside) {
      const float2 xk = xT[ti + 1][tj + 1];
      const float2 y = coarse_apply_tile(a, xT, ti, tj);
      const float2 d = fmul4(dk, make_float2(bk.x - y.x, bk.y - y.y));
      L.x[k] = make_float2(xk.x + omega * d.x, xk.y + omega * d.y);
    }
  }
}

// The small levels (first .. last) in one launch: restrictions down, the dense solve,
// post-smoothing up.
struct SmallLevels {
  int first, last;        // level indices into lev[]
  const LevelView *lev;   // device array of the level views (read through L1, no local copy)
  const double *invT;
  int n;                  // unknowns of the coarsest level
};

// the largest window (cells) any CTA stages in a cycle over levels first .. nlev - 1
inline int small_window_cells(const MGLevel *lev, int first, int nlev, int parts, int local_items) {
  int most = 0;
  for (int l = first; l + 1 < nlev; ++l) {
    const MGLevel &L = lev[l], &C = lev[l + 1];
    const int span = small_span(C.N), pd = span <= local_items ? 1 : parts;
    for (int c = 0; c < pd; ++c) {
      int b0, b1, r0, r1, w0, nr;
      small_chunk(span, pd, c, 32, b0, b1);
      if (b1 <= b0) continue;
      small_down_rows(L.ax, C.My, C.N, b0, b1, r0, r1);
      small_window(L.Mx, r0, r1, w0, nr);
      most = nr * L.My > most ? nr * L.My : most;
    }
    const int pu = L.N <= local_items ? 1 : parts;
    for (int c = 0; c < pu; ++c) {
      int k0, k1, w0, nr;
      small_chunk(L.N, pu, c, 32, k0, k1);
      if (k1 <= k0) continue;
      small_window(L.Mx, k0 / L.My, (k1 - 1) / L.My, w0, nr);
      most = nr * L.My > most ? nr * L.My : most;
    }
  }
  return most;
}

// The small levels run on one thread-block cluster of SMALL_CLUSTER CTAs: every CTA
// stages the rows its chunk of a step reads in its shared memory, computes its chunk, and the
// cluster barrier (release / acquire at cluster scope) orders the steps.

__global__ void __cluster_dims__(SMALL_CLUSTER, 1, 1) __launch_bounds__(CTA_THREADS)
    k_mg_small_cycle(SmallLevels S, float omega, float corr, const KState *st) {
  if (st && st->done) return;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = cluster.block_rank() * CTA_THREADS + threadIdx.x, nthr = SMALL_CLUSTER * CTA_THREADS;
  // the small levels' operators are evicted from L2 by the fine-level passes between
  // cycles; pull all of them back in at once instead of one dependent round per step
  for (int l = S.first; l <= S.last; ++l) {
    const LevelView L = S.lev[l];
    const char *A = reinterpret_cast<const char *>(L.A), *D = reinterpret_cast<const char *>(L.dinv);
    const int lines_A = (9 * L.N * (int)sizeof(float4) + 127) / 128, lines_D = (L.N * (int)sizeof(float4) + 127) / 128;
    for (int q = rank; q < lines_A + lines_D; q += nthr) {
      const char *p = q < lines_A ? A + 128 * (size_t)q : D + 128 * (size_t)(q - lines_A);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  }
  extern __shared__ float2 xs[];   // the largest window a CTA stages (H.small_smem bytes)
  __shared__ float bsh[2 * MG_MAX_COARSE_CELLS];
  // Each step below costs one dependent round trip to L2: the staging loops are unrolled so
  // a thread's loads issue together, and the restriction gives every fine cell of an
  // aggregate its own thread (four per coarse cell, summed by shuffles).  A step whose items
  // fit in one CTA (restrictions to levels of at most CTA_THREADS / 4 cells, the coarsest
  // solve, the post-smoothing of levels of at most CTA_THREADS cells) is CTA 0's alone and
  // ends with a CTA barrier instead of the cluster's; the other CTAs wait at one cluster
  // barrier for the first up step that needs them.  Every item is computed by the same
  // arithmetic whichever thread takes it, so the split does not change the results.
  const int part = cluster.block_rank();
  const bool lead = part == 0;
  // x at wrapped fine row ii of the staged window [w0, w0 + nrows)
  auto window = [&](int Mx, int My, int w0, int nrows) {
    return [=](int ii, int jj) {
      int r = ii - w0;
      if (r < 0) r += Mx;
      else if (r >= nrows) r -= Mx;
      return xs[r * My + jj];
    };
  };
  // down
  for (int l = S.first; l < S.last; ++l) {
    const LevelView L = S.lev[l], C = S.lev[l + 1];
    const int span = small_span(C.N);
    const bool local = span <= CTA_THREADS;
    if (local && !lead) break;
    int b0, b1;
    small_chunk(span, local ? 1 : SMALL_CLUSTER, local ? 0 : part, 32, b0, b1);
    if (b1 > b0) {
      int r0, r1, w0, nrows;
      small_down_rows(L.ax, C.My, C.N, b0, b1, r0, r1);
      small_window(L.Mx, r0, r1, w0, nrows);
#pragma unroll 4
      for (int q = threadIdx.x; q < nrows * L.My; q += CTA_THREADS) {
        const int r = q / L.My, j = q - r * L.My, k = pmod(w0 + r, L.Mx) * L.My + j;
        const float2 v = fmul4(L.dinv[k], L.b[k]);
        xs[q] = make_float2(omega * v.x, omega * v.y);
      }
      __syncthreads();
      const auto xa = window(L.Mx, L.My, w0, nrows);
      for (int base = b0 + threadIdx.x; base < b1; base += CTA_THREADS) {
        const int kc = base >> 2, pi = (base >> 1) & 1, pj = base & 1;
        float ru = 0.0f, rv = 0.0f;
        if (kc < C.N && pi < L.ax && pj < L.ay) {
          const int I = kc / C.My, J = kc - I * C.My;
          const int i = I * L.ax + pi, j = J * L.ay + pj;
          if (i < L.Mx && j < L.My) {
            const float2 y = coarse_apply(L, i, j, xa);
            const float2 bk = L.b[i * L.My + j];
            ru = bk.x - y.x;
            rv = bk.y - y.y;
          }
        }
        ru += __shfl_xor_sync(0xffffffffu, ru, 1);
        rv += __shfl_xor_sync(0xffffffffu, rv, 1);
        ru += __shfl_xor_sync(0xffffffffu, ru, 2);
        rv += __shfl_xor_sync(0xffffffffu, rv, 2);
        if (kc < C.N && (base & 3) == 0) C.b[kc] = make_float2(ru, rv);
      }
    }
    if (local) __syncthreads();
    else cluster.sync();
  }
  // coarsest: x = A^-1 b (S.n <= 32 rows: CTA 0's warps)
  if (lead) {
    const LevelView C = S.lev[S.last];
    for (int q = threadIdx.x; q < C.N; q += CTA_THREADS) {
      const float2 v = C.b[q];
      bsh[2 * q] = v.x;
      bsh[2 * q + 1] = v.y;
    }
    __syncthreads();
    // one warp per row, the lanes split the columns (the row-major transpose keeps a
    // column's entries of consecutive rows adjacent; here each lane reads its own column)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = CTA_THREADS >> 5;
    for (int r = warp; r < S.n; r += nwarp) {
      double acc = 0.0;
      for (int c = lane; c < S.n; c += 32) acc += S.invT[c * S.n + r] * (double)bsh[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) reinterpret_cast<float *>(C.x)[r] = (float)acc;
    }
    __syncthreads();
  }
  // up
  bool joined = false;   // the other CTAs are back (after CTA 0's levels)
  for (int l = S.last - 1; l >= S.first; --l) {
    const LevelView L = S.lev[l], C = S.lev[l + 1];
    const bool local = L.N <= CTA_THREADS;
    if (local && !lead) continue;
    if (!local && !joined) {
      cluster.sync();   // CTA 0's coarse levels are written
      joined = true;
    }
    int k0, k1;
    small_chunk(L.N, local ? 1 : SMALL_CLUSTER, local ? 0 : part, 32, k0, k1);
    if (k1 > k0) {
      int w0, nrows;
      small_window(L.Mx, k0 / L.My, (k1 - 1) / L.My, w0, nrows);
#pragma unroll 4
      for (int q = threadIdx.x; q < nrows * L.My; q += CTA_THREADS) {
        const int r = q / L.My, j = q - r * L.My, i = pmod(w0 + r, L.Mx), k = i * L.My + j;
        const float2 v = fmul4(L.dinv[k], L.b[k]);
        const float2 c = C.x[(i / L.ax) * C.My + j / L.ay];
        xs[q] = make_float2(omega * v.x + corr * c.x, omega * v.y + corr * c.y);
      }
      __syncthreads();
      const auto xa = window(L.Mx, L.My, w0, nrows);
      for (int k = k0 + threadIdx.x; k < k1; k += CTA_THREADS) {
        const int i = k / L.My, j = k - i * L.My;
        const float2 xk = xa(i, j);
        const float2 y = coarse_apply(L, i, j, xa);
        const float2 bk = L.b[k];
        const float2 d = fmul4(L.dinv[k], make_float2(bk.x - y.x, bk.y - y.y));
        L.x[k] = make_float2(xk.x + omega * d.x, xk.y + omega * d.y);
      }
    }
    if (local) __syncthreads();
    else cluster.sync();
  }
}

// ---------------------------------------------------------------------------
// The small levels in the cluster's shared memory.  Every CTA holds a nested block of every
// small level (ssa_small_plan.h): the nine 2 x 2 operator blocks and D^-1, staged once per
// cycle by bulk asynchronous copies (one per block row and array) completing on an
// mbarrier, and b, x0, x, z.  A step reads its own cells from its shared memory and the
// neighbours' halo values from the neighbouring CTAs' shared memory (distributed shared
// memory), so no step waits on L2; the restriction and the prolongation stay inside a CTA
// because the blocks nest.  The arithmetic of every cell is that of k_mg_small_cycle, in the
// same order, so the two give the same bits.
// ---------------------------------------------------------------------------
struct SmallDs {
  const SmallPlan *plan;   // device copy of the split
  const LevelView *lev;    // device level views
  int first;               // index of the first small level
  const double *invT;      // dense inverse of the coarsest operator (transposed)
  int n;                   // unknowns of the coarsest level
};

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// bounded wait for phase `phase` of an mbarrier: false when it did not complete
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned phase) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// y = A x at the cell with slot s of this CTA's block (level cells (i, j)), the nine blocks
// from shared memory, x through xf(i', j') (wrapped indices)
template <class XF>
__device__ __forceinline__ float2 small_apply(const float4 *__restrict__ A0, int cap, int s, int i, int j, int Mx,
                                              int My, const XF &xf) {
  const int ip = wrap(i + 1, Mx), im = wrap(i - 1, Mx), jp = wrap(j + 1, My), jm = wrap(j - 1, My);
  const int ii[9] = {im, i, ip, im, i, ip, im, i, ip};
  const int jj[9] = {jp, jp, jp, j, j, j, jm, jm, jm};
  float y1 = 0.0f, y2 = 0.0f;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const float4 a = A0[b * cap + s];
    const float2 xv = xf(ii[b], jj[b]);
    y1 += a.x * xv.x + a.y * xv.y;
    y2 += a.z * xv.x + a.w * xv.y;
  }
  return make_float2(y1, y2);
}

__global__ void __cluster_dims__(SMALL_CLUSTER, 1, 1) __launch_bounds__(CTA_THREADS)
    k_mg_small_dsmem(SmallDs S, float omega, float corr, KState *st) {
  if (st && st->done) return;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ SmallPlan P;
  __shared__ float bsh[2 * MG_MAX_COARSE_CELLS];
  __shared__ __align__(8) unsigned long long bar;
  const unsigned rank = cluster.block_rank();
  const int tid = threadIdx.x;
  for (int q = tid; q < (int)(sizeof(SmallPlan) / sizeof(int)); q += CTA_THREADS)
    reinterpret_cast<int *>(&P)[q] = reinterpret_cast<const int *>(S.plan)[q];
  __syncthreads();
  const int pr = (int)rank / P.Pc, pc = (int)rank % P.Pc;
  const bool active = (int)rank < P.Pr * P.Pc;
  auto cap = [&](int l) { return P.mi[l] * P.mj[l]; };
  // arrays of level l: blocks 0..8 of A and D^-1 (float4, cap slots each); b, z (float2, cap
  // slots each); x0, x (float2, padded: (mi + 2) x (mj + 2) with the halo ring)
  auto A4 = [&](int l) { return reinterpret_cast<float4 *>(sm + P.off4[l]); };
  auto F2 = [&](int l, int a) { return reinterpret_cast<float2 *>(sm + P.off2[l]) + a * cap(l); };
  auto PAD = [&](int l, int a) {
    return reinterpret_cast<float2 *>(sm + P.offp[l]) + a * (P.mi[l] + 2) * (P.mj[l] + 2);
  };
  auto r0 = [&](int l) { return active ? P.rb[l][pr] : 0; };
  auto c0 = [&](int l) { return active ? P.cb[l][pc] : 0; };
  auto ni = [&](int l) { return active ? P.rb[l][pr + 1] - P.rb[l][pr] : 0; };
  auto nj = [&](int l) { return active ? P.cb[l][pc + 1] - P.cb[l][pc] : 0; };
  // value of cell (ii, jj) (wrapped indices) of level l in the padded array `a` or, with
  // pad < 0, in the cap-slot array F2(l, -1 - pad), from whichever CTA holds it
  auto fetch_pad = [&](int l, int a, int ii, int jj) {
    const int qp = small_owner(P.rb[l], P.Pr, ii), qc = small_owner(P.cb[l], P.Pc, jj);
    const int s = (ii - P.rb[l][qp] + 1) * (P.mj[l] + 2) + (jj - P.cb[l][qc] + 1);
    float2 *base = PAD(l, a);
    const unsigned owner = (unsigned)(qp * P.Pc + qc);
    return owner == rank ? base[s] : cluster.map_shared_rank(base, owner)[s];
  };
  // the halo ring of this CTA's padded array `a` of level l, from the neighbours' interiors
  auto fill_ring = [&](int l, int a) {
    const int n_i = ni(l), n_j = nj(l), w = P.mj[l] + 2;
    const int top = n_j + 2, count = 2 * top + 2 * n_i;
    float2 *x = PAD(l, a);
    for (int t = tid; t < count; t += CTA_THREADS) {
      int pa, pb;   // padded coordinates
      if (t < top) {
        pa = 0;
        pb = t;
      } else if (t < 2 * top) {
        pa = n_i + 1;
        pb = t - top;
      } else if (t < 2 * top + n_i) {
        pa = t - 2 * top + 1;
        pb = 0;
      } else {
        pa = t - 2 * top - n_i + 1;
        pb = n_j + 1;
      }
      const int ii = pmod(r0(l) + pa - 1, P.Mx[l]), jj = pmod(c0(l) + pb - 1, P.My[l]);
      x[pa * w + pb] = fetch_pad(l, a, ii, jj);
    }
  };

  // ---- staging: this CTA's block of every level's operator by bulk copies, b of the first ----
  const unsigned bar_a = smem_addr(&bar);
  unsigned total = 0;
  for (int l = 0; l < P.nlev; ++l) total += (unsigned)(ni(l) * nj(l) * 10 * 16);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (total > 0)
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(total) : "memory");
  }
  __syncthreads();
  if (total > 0) {
    int nrow_total = 0;
    for (int l = 0; l < P.nlev; ++l) nrow_total += ni(l) * 10;
    for (int q = tid; q < nrow_total; q += CTA_THREADS) {
      int l = 0, rem = q;
      while (rem >= ni(l) * 10) {
        rem -= ni(l) * 10;
        ++l;
      }
      const int row = rem / 10, blk = rem - row * 10;
      const LevelView L = S.lev[S.first + l];
      const int i = r0(l) + row;
      const float4 *src = (blk < 9 ? L.A + (size_t)blk * L.N : L.dinv) + (size_t)i * L.My + c0(l);
      float4 *dst = A4(l) + blk * cap(l) + row * P.mj[l];
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(dst)),
          "l"(src), "r"((unsigned)(nj(l) * 16)), "r"(bar_a)
          : "memory");
    }
  }
  {
    const LevelView L = S.lev[S.first];
    float2 *b = F2(0, 0);
    for (int q = tid; q < ni(0) * nj(0); q += CTA_THREADS) {
      const int li = q / nj(0), lj = q - li * nj(0);
      b[li * P.mj[0] + lj] = L.b[(r0(0) + li) * L.My + c0(0) + lj];
    }
  }
  bool staged = true;
  if (total > 0) {
    staged = mbar_wait_bounded(bar_a, 0);
    if (!staged && tid == 0 && st) {   // the Krylov solve stops: this cycle ran on what had arrived
      st->done = 1;
      st->status = KSP_STALLED;
    }
  }
  __syncthreads();

  // ---- down: x0 = omega D^-1 b; b_{l+1} = R (b - A x0) ----
  for (int l = 0; l + 1 < P.nlev; ++l) {
    const int Mx = P.Mx[l], My = P.My[l], mj = P.mj[l], w = mj + 2, cp = cap(l);
    const float4 *A = A4(l), *D = A4(l) + 9 * cp;
    const float2 *b = F2(l, 0);
    float2 *x0 = PAD(l, 0);
    for (int q = tid; q < ni(l) * nj(l); q += CTA_THREADS) {
      const int li = q / nj(l), lj = q - li * nj(l), s = li * mj + lj;
      const float2 v = fmul4(D[s], b[s]);
      x0[(li + 1) * w + lj + 1] = make_float2(omega * v.x, omega * v.y);
    }
    cluster.sync();
    fill_ring(l, 0);
    __syncthreads();
    const int ax = P.ax[l], ay = P.ay[l], R0 = r0(l + 1), C0 = c0(l + 1), ncj = nj(l + 1), nc = ni(l + 1) * ncj;
    const int i0 = r0(l), j0 = c0(l);
    float2 *bc = F2(l + 1, 0);
    const int span = (4 * nc + 31) & ~31;   // whole warps take part in the shuffles
    for (int base = tid; base < span; base += CTA_THREADS) {
      const int kc = base >> 2, pi = (base >> 1) & 1, pj = base & 1;
      float ru = 0.0f, rv = 0.0f;
      if (kc < nc && pi < ax && pj < ay) {
        const int I = R0 + kc / ncj, J = C0 + kc % ncj;
        const int i = I * ax + pi, j = J * ay + pj;
        if (i < Mx && j < My) {
          const int li = i - i0, lj = j - j0, s = li * mj + lj;
          const float2 y = small_apply(A, cp, s, i, j, Mx, My, [&](int ii, int jj) {
            // (ii, jj) is a neighbour of (i, j): its padded position from the offset
            return x0[(li + 1 + wdiff(ii, i, Mx)) * w + (lj + 1 + wdiff(jj, j, My))];
          });
          const float2 bk = b[s];
          ru = bk.x - y.x;
          rv = bk.y - y.y;
        }
      }
      ru += __shfl_xor_sync(0xffffffffu, ru, 1);
      rv += __shfl_xor_sync(0xffffffffu, rv, 1);
      ru += __shfl_xor_sync(0xffffffffu, ru, 2);
      rv += __shfl_xor_sync(0xffffffffu, rv, 2);
      if (kc < nc && (base & 3) == 0) bc[(kc / ncj) * P.mj[l + 1] + kc % ncj] = make_float2(ru, rv);
    }
    __syncthreads();
  }

  // ---- coarsest: x = A^-1 b (every CTA gathers b, each computes the rows of its cells) ----
  {
    const int l = P.nlev - 1, Myc = P.My[l], Nc = P.Mx[l] * Myc;
    cluster.sync();
    for (int q = tid; q < Nc; q += CTA_THREADS) {
      const int ii = q / Myc, jj = q % Myc;
      const int qp = small_owner(P.rb[l], P.Pr, ii), qc = small_owner(P.cb[l], P.Pc, jj);
      const int s = (ii - P.rb[l][qp]) * P.mj[l] + (jj - P.cb[l][qc]);
      const unsigned owner = (unsigned)(qp * P.Pc + qc);
      float2 *base = F2(l, 0);
      const float2 v = owner == rank ? base[s] : cluster.map_shared_rank(base, owner)[s];
      bsh[2 * q] = v.x;
      bsh[2 * q + 1] = v.y;
    }
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5, nrows = 2 * ni(l) * nj(l);
    float *z = reinterpret_cast<float *>(F2(l, 1));
    const LevelView Lc = S.lev[S.first + l];
    for (int wv = warp; wv < nrows; wv += CTA_THREADS / 32) {
      const int q = wv >> 1, comp = wv & 1, li = q / nj(l), lj = q - li * nj(l);
      const int r = 2 * ((r0(l) + li) * Myc + c0(l) + lj) + comp;
      double acc = 0.0;
      for (int c = lane; c < S.n; c += 32) acc += S.invT[c * S.n + r] * (double)bsh[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) {
        z[2 * (li * P.mj[l] + lj) + comp] = (float)acc;
        if (P.nlev == 1) reinterpret_cast<float *>(Lc.x)[r] = (float)acc;
      }
    }
    __syncthreads();
  }

  // ---- up: x = omega D^-1 b + s P z_{l+1}; z = x + omega D^-1 (b - A x) ----
  for (int l = P.nlev - 2; l >= 0; --l) {
    const int Mx = P.Mx[l], My = P.My[l], mj = P.mj[l], w = mj + 2, cp = cap(l);
    const float4 *A = A4(l), *D = A4(l) + 9 * cp;
    const float2 *b = F2(l, 0), *zc = F2(l + 1, 1);
    float2 *x = PAD(l, 1), *z = F2(l, 1);
    const int ax = P.ax[l], ay = P.ay[l], R0 = r0(l + 1), C0 = c0(l + 1), mjc = P.mj[l + 1];
    for (int q = tid; q < ni(l) * nj(l); q += CTA_THREADS) {
      const int li = q / nj(l), lj = q - li * nj(l), s = li * mj + lj;
      const int i = r0(l) + li, j = c0(l) + lj;
      const float2 v = fmul4(D[s], b[s]);
      const float2 c = zc[(i / ax - R0) * mjc + (j / ay - C0)];
      x[(li + 1) * w + lj + 1] = make_float2(omega * v.x + corr * c.x, omega * v.y + corr * c.y);
    }
    cluster.sync();
    fill_ring(l, 1);
    __syncthreads();
    const LevelView L = S.lev[S.first + l];
    for (int q = tid; q < ni(l) * nj(l); q += CTA_THREADS) {
      const int li = q / nj(l), lj = q - li * nj(l), s = li * mj + lj;
      const int i = r0(l) + li, j = c0(l) + lj;
      const float2 xk = x[(li + 1) * w + lj + 1];
      const float2 y = small_apply(A, cp, s, i, j, Mx, My, [&](int ii, int jj) {
        return x[(li + 1 + wdiff(ii, i, Mx)) * w + (lj + 1 + wdiff(jj, j, My))];
      });
      const float2 bk = b[s];
      const float2 d = fmul4(D[s], make_float2(bk.x - y.x, bk.y - y.y));
      const float2 zk = make_float2(xk.x + omega * d.x, xk.y + omega * d.y);
      z[s] = zk;
      if (l == 0) L.x[i * My + j] = zk;
    }
    __syncthreads();
  }
  // no CTA leaves while another may still read its shared memory; after a staging wait
  // that gave up, the copies still in flight are waited for once more (bounded) first
  if (!staged) mbar_wait_bounded(bar_a, 0);
  cluster.sync();
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int mg_plan(int Mx, int My, MGHierarchy &H) {
  H.nlev = 0;
  int mx = Mx, my = My;
  if (mx <= MG_COARSE_DIM && my <= MG_COARSE_DIM) return 0;   // too small for a hierarchy
  H.fine_ax = mx > MG_COARSE_DIM ? 2 : 1;
  H.fine_ay = my > MG_COARSE_DIM ? 2 : 1;
  mx = (mx + H.fine_ax - 1) / H.fine_ax;
  my = (my + H.fine_ay - 1) / H.fine_ay;
  while (H.nlev < MG_MAX_LEVELS) {
    MGLevel &L = H.lev[H.nlev++];
    L.Mx = mx;
    L.My = my;
    L.N = mx * my;
    if (mx <= MG_COARSE_DIM && my <= MG_COARSE_DIM) break;
    L.ax = mx > MG_COARSE_DIM ? 2 : 1;
    L.ay = my > MG_COARSE_DIM ? 2 : 1;
    mx = (mx + L.ax - 1) / L.ax;
    my = (my + L.ay - 1) / L.ay;
  }
  MGLevel &C = H.lev[H.nlev - 1];
  if (C.Mx > MG_COARSE_DIM || C.My > MG_COARSE_DIM) {   // ran out of levels
    H.nlev = 0;
    return 0;
  }
  C.ax = C.ay = 1;
  // the levels cycled by the cluster kernel: the trailing run of levels with <= MG_CTA_CELLS cells
  H.small_first = H.nlev - 1;
  while (H.small_first > 0 && H.lev[H.small_first - 1].N <= MG_CTA_CELLS) --H.small_first;
  // mg_small_kernel 2: the trailing run of levels with <= MG_CTA_CELLS_WIDE cells
  H.small_first_wide = H.small_first;
  while (H.small_first_wide > 0 && H.lev[H.small_first_wide - 1].N <= MG_CTA_CELLS_WIDE) --H.small_first_wide;
  // every CTA stages the rows its share of a step reads
  H.small_smem = (int)sizeof(float2) *
                 std::max(small_window_cells(H.lev, H.small_first, H.nlev, SMALL_CLUSTER, CTA_THREADS),
                          small_window_cells(H.lev, H.small_first_wide, H.nlev, SMALL_CLUSTER, CTA_THREADS));
  // the shared-memory cycle when every small level's block fits (ssa_small_plan.h)
  {
    int mx[SC_MAX_LEV], my[SC_MAX_LEV], ax[SC_MAX_LEV], ay[SC_MAX_LEV];
    const int ns = H.nlev - H.small_first;
    H.small_dsmem = false;
    if (ns <= SC_MAX_LEV) {
      for (int l = 0; l < ns; ++l) {
        const MGLevel &L = H.lev[H.small_first + l];
        mx[l] = L.Mx;
        my[l] = L.My;
        ax[l] = L.ax;
        ay[l] = L.ay;
      }
      H.small_dsmem = small_plan(ns, mx, my, ax, ay, SMALL_DSMEM_MAX_BYTES, H.small_plan);
    }
  }
  return H.nlev;
}

// The dynamic shared-memory limit of a kernel is an attribute of the function on the current
// device, shared by every handle of the process: a handle on a smaller grid must not lower the
// limit that a live handle on a larger grid launches with.  So the attribute is only ever
// raised, to the largest size any handle has asked for on that device (under a lock: handles
// may be created from several host threads).
static int raise_dynamic_smem(const void *func, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, int> granted;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  std::lock_guard<std::mutex> lock(mu);
  int &have = granted[{dev, func}];
  if (bytes <= have) return 0;
  if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) return 1;
  have = bytes;
  return 0;
}

int mg_allocate(MGHierarchy &H, int fine_cells) {
  for (int l = 0; l < H.nlev; ++l) {
    MGLevel &L = H.lev[l];
    if (cudaMalloc(&L.A, sizeof(float4) * 9 * L.N) != cudaSuccess) return 1;
    if (cudaMalloc(&L.dinv, sizeof(float4) * L.N) != cudaSuccess) return 1;
    if (cudaMalloc(&L.b, sizeof(float2) * L.N) != cudaSuccess) return 1;
    if (cudaMalloc(&L.x, sizeof(float2) * L.N) != cudaSuccess) return 1;
  }
  if (cudaMalloc(&H.nuHf, sizeof(float2) * fine_cells) != cudaSuccess) return 1;
  if (cudaMalloc(&H.betaf, sizeof(float) * fine_cells) != cudaSuccess) return 1;
  if (cudaMalloc(&H.dinvf, sizeof(float4) * fine_cells) != cudaSuccess) return 1;
  const int n = 2 * H.lev[H.nlev - 1].N;
  if (cudaMalloc(&H.cinv, sizeof(double) * n * n) != cudaSuccess) return 1;
  if (cudaMalloc(&H.singular, sizeof(int)) != cudaSuccess) return 1;
  {
    LevelView v[MG_MAX_LEVELS];
    for (int l = 0; l < H.nlev; ++l)
      v[l] = LevelView{H.lev[l].Mx, H.lev[l].My, H.lev[l].N, H.lev[l].ax, H.lev[l].ay, H.lev[l].A, H.lev[l].dinv,
                       H.lev[l].b, H.lev[l].x};
    if (cudaMalloc(&H.views, sizeof(LevelView) * MG_MAX_LEVELS) != cudaSuccess) return 1;
    if (cudaMemcpy(H.views, v, sizeof(LevelView) * H.nlev, cudaMemcpyHostToDevice) != cudaSuccess) return 1;
  }
  if (raise_dynamic_smem((const void *)k_mg_small_cycle, H.small_smem) != 0) return 1;
  if (H.small_dsmem) {
    if (cudaMalloc(&H.small_plan_dev, sizeof(SmallPlan)) != cudaSuccess) return 1;
    if (cudaMemcpy(H.small_plan_dev, &H.small_plan, sizeof(SmallPlan), cudaMemcpyHostToDevice) != cudaSuccess)
      return 1;
    if (raise_dynamic_smem((const void *)k_mg_small_dsmem, H.small_plan.smem) != 0) return 1;
  }
  return 0;
}

void mg_free(MGHierarchy &H) {
  for (int l = 0; l < MG_MAX_LEVELS; ++l) {
    MGLevel &L = H.lev[l];
    cudaFree(L.A);
    cudaFree(L.dinv);
    cudaFree(L.b);
    cudaFree(L.x);
    L.A = nullptr;
    L.dinv = nullptr;
    L.b = L.x = nullptr;
  }
  cudaFree(H.nuHf);
  cudaFree(H.betaf);
  cudaFree(H.dinvf);
  cudaFree(H.cinv);
  cudaFree(H.singular);
  cudaFree(H.views);
  cudaFree(H.small_plan_dev);
  H.small_plan_dev = nullptr;
  H.views = nullptr;
  H.nuHf = nullptr;
  H.betaf = nullptr;
  H.dinvf = nullptr;
  H.cinv = nullptr;
  H.singular = nullptr;
  H.nlev = 0;
}

static LevelView view(const MGLevel &L) { return LevelView{L.Mx, L.My, L.N, L.ax, L.ay, L.A, L.dinv, L.b, L.x}; }

static int blocks_for(const Launch &Lc, int tiles) { return std::min(tiles, Lc.max_blocks); }

FineF fine_view(const GridDev &g, const Fields &f, const MGHierarchy &H) {
  FineF F;
  F.g = g;
  F.rdx2 = (float)(1.0 / (g.dx * g.dx));
  F.rdy2 = (float)(1.0 / (g.dy * g.dy));
  F.r2 = (float)(1.0 / (2 * g.dx * g.dy));
  F.r4 = (float)(1.0 / (4 * g.dx * g.dy));
  F.scaling = 1.0e9f;
  F.nu_bedrock = (float)f.nu_bedrock;
  F.flags = f.flags;
  F.nuH = H.nuHf;
  F.beta = H.betaf;
  F.dinv = H.dinvf;
  F.H = f.H;
  return F;
}

void mg_setup(const Launch &Lc, const GridDev &g, const Fields &f, const double4 *dinv0, MGHierarchy &H) {
  mg_setup_fine(Lc, g, f, dinv0, H);
  mg_setup_coarse(Lc, g, f, H);
}

// the FP32 fine-level copies of nu*H, beta and D^-1 (the smoother's and the FP32 Krylov
// operator's): always from the current nu*H
void mg_setup_fine(const Launch &Lc, const GridDev &g, const Fields &f, const double4 *dinv0, MGHierarchy &H) {
  const int N = g.Mx * g.My;
  k_mg0_compact<<<std::min((N + NTm - 1) / NTm, Lc.max_blocks), NTm, 0, Lc.stream>>>(N, f.nuH, f.beta, dinv0, H.nuHf,
                                                                                     H.betaf, H.dinvf);
  Lc.tick();
}

// the coarse levels: Galerkin operators and D^-1 of every level, the coarsest inverse
void mg_setup_coarse(const Launch &Lc, const GridDev &g, const Fields &f, MGHierarchy &H) {
  const StencilConst s = stencil_const(g, f);
  {
    const MGLevel &C = H.lev[0];
    const TileM tm = tiles_of(C.Mx, C.My);
    k_mg_build1<<<blocks_for(Lc, tm.tiles), NTm, 0, Lc.stream>>>(g, s, f.flags, f.nuH, f.beta, H.fine_ax,
                                                                     H.fine_ay, C.Mx, C.My, tm, C.A, C.dinv);
  }
  // levels 1 .. cfirst - 1 by tiled passes; cfirst .. nlev - 1 (the cluster-cycled small
  // levels) by one cluster launch; then the coarsest inverse
  const int cfirst = H.nlev > 1 ? std::max(1, H.small_first) : H.nlev;
  for (int l = 0; l + 1 < cfirst; ++l) {
    const MGLevel &F = H.lev[l], &C = H.lev[l + 1];
    const TileM tm = tiles_of(C.Mx, C.My);
    k_mg_build<<<blocks_for(Lc, tm.tiles), NTm, 0, Lc.stream>>>(view(F), C.Mx, C.My, tm, C.A, C.dinv);
  }
  if (cfirst < H.nlev) {
    k_mg_build_small<<<SMALL_CLUSTER, NTm, 0, Lc.stream>>>(reinterpret_cast<const LevelView *>(H.views), cfirst,
                                                             H.nlev);
    Lc.tick();
  }
  k_mg_coarse_invert<<<1, CI_THREADS, 0, Lc.stream>>>(view(H.lev[H.nlev - 1]), H.cinv, H.singular);
  Lc.tick(cfirst + 1);
}

template <class F22, class F21, class F12, class F11>
static void dispatch_ax(int ax, int ay, F22 f22, F21 f21, F12 f12, F11 f11) {
  if (ax == 2 && ay == 2) f22();
  else if (ax == 2) f21();
  else if (ay == 2) f12();
  else f11();
}

struct NoEpi {};

// One V-cycle z = M^-1 b; with an epilogue EPI (EpiV, EpiT) the fine-level pass also applies A
// to z and hands y = A z to it (k_mg0_post_apply)
template <class BA, class ZV, class EPI = NoEpi>
static void vcycle(const Launch &Lc, const GridDev &g, const Fields &f, const MGHierarchy &H, BA b, ZV *z,
                   KState *st, const EPI &epi = EPI{}) {
  const FineF F = fine_view(g, f, H);
  const float omega = H.omega, corr = H.correction;
  int launches = 0;
  // down: fine -> level 1
  {
    const MGLevel &C = H.lev[0];
    const TileM tm = tiles_of(g.Mx, g.My);
    const int nb = blocks_for(Lc, tm.tiles);
#define MG0R(AX, AY) [&] { k_mg0_restrict<AX, AY, BA><<<nb, NTm, 0, Lc.stream>>>(F, b, omega, C.Mx, C.My, tm, C.b, st); }
    dispatch_ax(H.fine_ax, H.fine_ay, MG0R(2, 2), MG0R(2, 1), MG0R(1, 2), MG0R(1, 1));
#undef MG0R
    ++launches;
  }
  // down through the large coarse levels
  // the first level the cluster cycles (mg_small_kernel 2: the wider set)
  const bool dsmem = H.small_dsmem && H.small_kernel == 1;
  const int first = H.small_kernel == 2 ? H.small_first_wide : H.small_first;
  for (int l = 0; l < first; ++l) {
    const MGLevel &L = H.lev[l], &C = H.lev[l + 1];
    const LevelView V = view(L);
    const TileM tm = tiles_of(L.Mx, L.My);
    const int nb = blocks_for(Lc, tm.tiles);
#define MGCR(AX, AY) [&] { k_mgc_restrict<AX, AY><<<nb, NTm, 0, Lc.stream>>>(V, omega, C.Mx, C.My, tm, C.b, st); }
    dispatch_ax(L.ax, L.ay, MGCR(2, 2), MGCR(2, 1), MGCR(1, 2), MGCR(1, 1));
#undef MGCR
    ++launches;
  }
  // the small levels on one thread-block cluster
  if (dsmem) {
    SmallDs S;
    S.plan = reinterpret_cast<const SmallPlan *>(H.small_plan_dev);
    S.lev = reinterpret_cast<const LevelView *>(H.views);
    S.first = H.small_first;
    S.invT = H.cinv;
    S.n = 2 * H.lev[H.nlev - 1].N;
    k_mg_small_dsmem<<<SMALL_CLUSTER, CTA_THREADS, H.small_plan.smem, Lc.stream>>>(S, omega, corr, st);
    ++launches;
  } else {
    SmallLevels S;
    S.first = first;
    S.last = H.nlev - 1;
    S.lev = reinterpret_cast<const LevelView *>(H.views);
    S.invT = H.cinv;
    S.n = 2 * H.lev[H.nlev - 1].N;
    k_mg_small_cycle<<<SMALL_CLUSTER, CTA_THREADS, H.small_smem, Lc.stream>>>(S, omega, corr, st);
    ++launches;
  }
  // up through the large coarse levels
  for (int l = first - 1; l >= 0; --l) {
    const MGLevel &L = H.lev[l], &C = H.lev[l + 1];
    const LevelView V = view(L);
    const TileM tm = tiles_of(L.Mx, L.My);
    const int nb = H.post_blocks > 0 ? std::min(blocks_for(Lc, tm.tiles), H.post_blocks) : blocks_for(Lc, tm.tiles);
#define MGCP(AX, AY) [&] { k_mgc_post<AX, AY><<<nb, NTm, 0, Lc.stream>>>(V, omega, corr, C.My, C.x, tm, st); }
    dispatch_ax(L.ax, L.ay, MGCP(2, 2), MGCP(2, 1), MGCP(1, 2), MGCP(1, 1));
#undef MGCP
    ++launches;
  }
  // fine level
  {
    const MGLevel &C = H.lev[0];
    const TileM tm = tiles_of(g.Mx, g.My);
    const int nb = blocks_for(Lc, tm.tiles);
    if constexpr (std::is_same<EPI, NoEpi>::value) {
#define MG0P(AX, AY) [&] { k_mg0_post<AX, AY, BA, ZV><<<nb, NTm, 0, Lc.stream>>>(F, b, omega, corr, C.My, C.x, tm, z, st); }
      dispatch_ax(H.fine_ax, H.fine_ay, MG0P(2, 2), MG0P(2, 1), MG0P(1, 2), MG0P(1, 1));
#undef MG0P
    } else {
      static_assert(std::is_same<ZV, float2>::value, "the fused pass produces FP32 iterates");
#define MG0PA(AX, AY) [&] { k_mg0_post_apply<AX, AY, BA, EPI><<<nb, NTm, 0, Lc.stream>>>(F, b, omega, corr, C.My, C.x, tm, z, epi); }
      dispatch_ax(H.fine_ax, H.fine_ay, MG0PA(2, 2), MG0PA(2, 1), MG0PA(1, 2), MG0PA(1, 1));
#undef MG0PA
    }
    ++launches;
  }
  Lc.tick(launches);
}

void mg_vcycle(const Launch &Lc, const GridDev &g, const Fields &f, const MGHierarchy &H, const double2 *b, double2 *z,
               KState *st) {
  vcycle(Lc, g, f, H, VecAcc<double2>{b}, z, st);
}

void mg_vcycle(const Launch &Lc, const GridDev &g, const Fields &f, const MGHierarchy &H, const float2 *b, float2 *z,
               KState *st) {
  vcycle(Lc, g, f, H, VecAcc<float2>{b}, z, st);
}

void mg_vcycle_s(const Launch &Lc, const GridDev &g, const Fields &f, const MGHierarchy &H, const float2 *r,
                 const float2 *v, float2 *z, KState *st) {
  vcycle(Lc, g, f, H, SAcc{r, v, st, 0.0f}, z, st);
}

void mg_vcycle_apply(const Launch &Lc, const GridDev &g, const Fields &f, const MGHierarchy &H, const float2 *b,
                     float2 *z, const EpiV &e) {
  vcycle(Lc, g, f, H, VecAcc<float2>{b}, z, e.st, e);
}

void mg_vcycle_s_apply(const Launch &Lc, const GridDev &g, const Fields &f, const MGHierarchy &H, const float2 *r,
                       const float2 *v, float2 *z, const EpiT &e) {
  vcycle(Lc, g, f, H, SAcc{r, v, e.st, 0.0f}, z, e.st, e);
}

}  // namespace pism_gpu
