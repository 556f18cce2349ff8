// ssa_line.cu — line block-Jacobi preconditioner for the SSAFD system.
//
// M is the part of the SSAFD matrix (SSAFD::assemble_matrix, SSAFD.cc:496-811) that couples
// each cell to itself and to its neighbours j - 1 and j + 1 on the same grid line of
// constant i (j is the contiguous axis).  Couplings between lines, and the two across a
// line's ends (the periodic wrap included), are dropped.  Each line's 2 x 2-block
// tridiagonal system is solved exactly; this stands in for the reference's default block
// Jacobi / ILU(0) preconditioner (SSAFD.cc:136-161), whose triangular solves run
// sequentially over the whole subdomain.
//
// Set-up, once per Picard iteration after nu*H and beta:
//   k_line_blocks   per cell: the blocks D (self), L (j - 1) and U (j + 1) of its two rows
//   k_line_factor   per line, sequential in j: block LU with P_j = (D_j - L_j G_{j-1})^-1,
//                   F_j = -P_j L_j, G_j = P_j U_j.  A pivot block that cannot be inverted
//                   restarts the line there (L_j dropped, P_j = D_j^-1 from block Jacobi).
// Apply, z = M^-1 r, one thread block per line:
//   forward   y_j = P_j r_j + F_j y_{j-1}
//   backward  x_j = y_j - G_j x_{j+1}
// Both are first-order linear recurrences y_j = M_j y_{j-1} + a_j.  The block solves 256
// cells at once with an inclusive scan over the affine maps (M_j, a_j), composed as
// (M2, a2) o (M1, a1) = (M2 M1, M2 a1 + a2) — the parallel-prefix form of a linear
// recurrence (Kogge and Stone, IEEE Trans. Computers C-22, 1973) — and carries y from one
// chunk of 256 cells to the next.
//
// Bytes per cell and apply: r, P, F, y (forward), y, G, x (backward) = 160 B in FP64.
#include "ssa_internal.h"
#include "ssa_stencil.cuh"

namespace pism_gpu {
namespace {

constexpr int LINE_THREADS = 256;   // cells of a line solved at once by the apply
constexpr int FACTOR_THREADS = 32;  // lines per block of the sequential factorisation
constexpr int FACTOR_AHEAD = 4;     // cells loaded ahead of the factorisation's recurrence

__device__ __forceinline__ double4 zero4() { return make_double4(0.0, 0.0, 0.0, 0.0); }

// 2 x 2 blocks as double4 (a11, a12, a21, a22)
__device__ __forceinline__ double4 mmul(const double4 &a, const double4 &b) {
  return make_double4(a.x * b.x + a.y * b.z, a.x * b.y + a.y * b.w, a.z * b.x + a.w * b.z, a.z * b.y + a.w * b.w);
}
__device__ __forceinline__ double4 msub(const double4 &a, const double4 &b) {
  return make_double4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
__device__ __forceinline__ double4 mneg(const double4 &a) { return make_double4(-a.x, -a.y, -a.z, -a.w); }
__device__ __forceinline__ bool minv(const double4 &a, double4 &out) {
  const double det = a.x * a.w - a.y * a.z;
  if (!(det != 0.0) || !isfinite(det)) return false;
  const double r = 1.0 / det;
  if (!isfinite(r)) return false;
  out = make_double4(a.w * r, -a.y * r, -a.z * r, a.x * r);
  return true;
}

struct Affine {   // y -> M y + a
  double4 M;
  double2 a;
};

// `first`, then `then`
__device__ __forceinline__ Affine compose(const Affine &first, const Affine &then) {
  Affine r;
  r.M = mmul(then.M, first.M);
  const double2 t = dmul(then.M, first.a);
  r.a = make_double2(t.x + then.a.x, t.y + then.a.y);
  return r;
}

__device__ __forceinline__ Affine shfl_up(const Affine &e, int d) {
  Affine o;
  o.M.x = __shfl_up_sync(0xffffffffu, e.M.x, d);
  o.M.y = __shfl_up_sync(0xffffffffu, e.M.y, d);
  o.M.z = __shfl_up_sync(0xffffffffu, e.M.z, d);
  o.M.w = __shfl_up_sync(0xffffffffu, e.M.w, d);
  o.a.x = __shfl_up_sync(0xffffffffu, e.a.x, d);
  o.a.y = __shfl_up_sync(0xffffffffu, e.a.y, d);
  return o;
}

// inclusive scan of the block's maps in thread order (warp scans, then the warp totals)
__device__ __forceinline__ Affine block_scan(Affine e, Affine *wtot) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Affine o = shfl_up(e, d);
    if (lane >= d) e = compose(o, e);
  }
  if (lane == 31) wtot[w] = e;
  __syncthreads();
  if (w > 0) {
    Affine pre = wtot[0];
    for (int q = 1; q < w; ++q) pre = compose(pre, wtot[q]);
    e = compose(pre, e);
  }
  return e;
}

// the in-line blocks of every cell's two rows (stencil_rows: N = j + 1, S = j - 1)
__global__ void __launch_bounds__(256) k_line_blocks(GridDev g, StencilConst s, const uint32_t *__restrict__ flags,
                                                     const double2 *__restrict__ nuH, const double *__restrict__ beta,
                                                     double4 *__restrict__ D, double4 *__restrict__ Lo,
                                                     double4 *__restrict__ Up) {
  const int N = g.Mx * g.My;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const int i = k / g.My, j = k - i * g.My;
    Row2 e1, e2;
    if (!cell_rows(g, s, i, j, flags[k], nuH, beta, e1, e2)) {   // Dirichlet / CFBC ice-free row
      D[k] = make_double4(s.scaling, 0.0, 0.0, s.scaling);
      Lo[k] = zero4();
      Up[k] = zero4();
      continue;
    }
    D[k] = make_double4(e1.uC, e1.vC, e2.uC, e2.vC);
    Lo[k] = j > 0 ? make_double4(e1.uS, e1.vS, e2.uS, e2.vS) : zero4();
    Up[k] = j < g.My - 1 ? make_double4(e1.uN, e1.vN, e2.uN, e2.vN) : zero4();
  }
}

// Block LU of each line, in place: P holds D on entry, F holds L, G holds U.  One thread
// per line; the next FACTOR_AHEAD cells' blocks are loaded while the recurrence runs.
__global__ void __launch_bounds__(FACTOR_THREADS) k_line_factor(GridDev g, const double4 *__restrict__ dinv,
                                                                double4 *P, double4 *F, double4 *G) {
  const int My = g.My;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.Mx; i += gridDim.x * blockDim.x) {
    const size_t row = (size_t)i * My;
    double4 bD[FACTOR_AHEAD], bL[FACTOR_AHEAD], bU[FACTOR_AHEAD];
#pragma unroll
    for (int q = 0; q < FACTOR_AHEAD; ++q)
      if (q < My) {
        bD[q] = P[row + q];
        bL[q] = F[row + q];
        bU[q] = G[row + q];
      }
    double4 Gp = zero4();
    for (int j0 = 0; j0 < My; j0 += FACTOR_AHEAD) {
#pragma unroll
      for (int q = 0; q < FACTOR_AHEAD; ++q) {
        const int j = j0 + q;
        if (j < My) {
          const size_t k = row + j;
          const double4 D = bD[q], Lb = bL[q], U = bU[q];
          if (j + FACTOR_AHEAD < My) {
            bD[q] = P[k + FACTOR_AHEAD];
            bL[q] = F[k + FACTOR_AHEAD];
            bU[q] = G[k + FACTOR_AHEAD];
          }
          double4 Pinv, Lk = Lb;
          if (!minv(msub(D, mmul(Lb, Gp)), Pinv)) {
            Pinv = dinv[k];
            Lk = zero4();
          }
          const double4 Gk = mmul(Pinv, U);
          P[k] = Pinv;
          F[k] = mneg(mmul(Pinv, Lk));
          G[k] = Gk;
          Gp = Gk;
        }
      }
    }
  }
}

// z = M^-1 b; b and z must not overlap
__global__ void __launch_bounds__(LINE_THREADS) k_line_apply(GridDev g, const double4 *__restrict__ P,
                                                             const double4 *__restrict__ F,
                                                             const double4 *__restrict__ G,
                                                             const double2 *__restrict__ b, double2 *z,
                                                             const KState *st) {
  if (st && st->done) return;
  __shared__ Affine wtot[LINE_THREADS / 32];
  __shared__ double2 carry;
  const int My = g.My, t = threadIdx.x;
  const int chunks = (My + LINE_THREADS - 1) / LINE_THREADS;
  Affine id;
  id.M = make_double4(1.0, 0.0, 0.0, 1.0);
  id.a = make_double2(0.0, 0.0);
  for (int i = blockIdx.x; i < g.Mx; i += gridDim.x) {
    const size_t row = (size_t)i * My;
    double2 cy = make_double2(0.0, 0.0);
    for (int c = 0; c < chunks; ++c) {   // forward, cells in thread order
      const int j = c * LINE_THREADS + t;
      Affine e = id;
      if (j < My) {
        e.M = F[row + j];
        e.a = dmul(P[row + j], b[row + j]);
      }
      e = block_scan(e, wtot);
      const double2 m = dmul(e.M, cy);
      const double2 y = make_double2(m.x + e.a.x, m.y + e.a.y);
      if (j < My) z[row + j] = y;
      if (t == LINE_THREADS - 1) carry = y;   // the chunk's last cell (padding maps are identities)
      __syncthreads();
      cy = carry;
    }
    cy = make_double2(0.0, 0.0);
    for (int c = chunks - 1; c >= 0; --c) {   // backward, cells in reverse thread order
      const int j0 = c * LINE_THREADS, j1 = min(My, j0 + LINE_THREADS), j = j1 - 1 - t;
      Affine e = id;
      if (j >= j0) {
        e.M = mneg(G[row + j]);
        e.a = z[row + j];
      }
      e = block_scan(e, wtot);
      const double2 m = dmul(e.M, cy);
      const double2 x = make_double2(m.x + e.a.x, m.y + e.a.y);
      if (j >= j0) z[row + j] = x;
      if (t == LINE_THREADS - 1) carry = x;   // the chunk's first cell
      __syncthreads();
      cy = carry;
    }
  }
}

}  // namespace

void line_setup(const Launch &L, const GridDev &g, const Fields &f, const double4 *dinv, const LinePC &lp) {
  L.tick(2);
  const int N = g.Mx * g.My;
  int nb = (N + 255) / 256;
  if (nb > L.max_blocks) nb = L.max_blocks;
  k_line_blocks<<<nb, 256, 0, L.stream>>>(g, stencil_const(g, f), f.flags, f.nuH, f.beta, lp.P, lp.F, lp.G);
  k_line_factor<<<(g.Mx + FACTOR_THREADS - 1) / FACTOR_THREADS, FACTOR_THREADS, 0, L.stream>>>(g, dinv, lp.P, lp.F,
                                                                                               lp.G);
}

void line_apply(const Launch &L, const GridDev &g, const LinePC &lp, const double2 *b, double2 *z,
                const KState *st) {
  L.tick();
  const int nb = g.Mx < 4 * L.max_blocks ? g.Mx : 4 * L.max_blocks;
  k_line_apply<<<nb, LINE_THREADS, 0, L.stream>>>(g, lp.P, lp.F, lp.G, b, z, st);
}

}  // namespace pism_gpu
