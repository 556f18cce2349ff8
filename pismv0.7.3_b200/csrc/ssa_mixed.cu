// ssa_mixed.cu — the mixed-precision linear solve: FP64 iterative refinement around an FP32
// BiCGStab preconditioned by the (FP32) multigrid V-cycle.
//
//   r = b - A x            FP64 operator, FP64 vectors; stop when ||r|| <= rtol ||b||
//   A d = r  (approx.)     FP32 operator from FP32 nu*H / beta, FP32 vectors, FP64 dots;
//                          to the relative tolerance mixed_inner_rtol
//   x <- x + d             FP64
//
// The outer residual, the convergence test and the solution stay FP64, so the accepted
// answer meets the same ||b - A x|| <= rtol ||b|| as the plain FP64 solve; the FP32 stencil
// reads 32 B per cell (x 8, nu*H 8, beta 4, flags 4, y 8) instead of 60.
#include "ssa_fine32.cuh"
#include "ssa_krylov32.cuh"
#include "ssa_tma_tile.cuh"

namespace pism_gpu {

namespace {

constexpr int NT32 = TILE_THREADS;

struct Tile32 {
  int tiles_j, tiles;
};

Tile32 tiles32(const GridDev &g) {
  Tile32 t;
  t.tiles_j = (g.My + TILE_J - 1) / TILE_J;
  t.tiles = t.tiles_j * ((g.Mx + TILE_I - 1) / TILE_I);
  return t;
}

// y = A x at this thread's cell of tile t (FP32); false outside the grid
// (the cell's flags and beta are issued with the tile loads: one round trip per tile)
__device__ __forceinline__ bool apply32(const FineF &F, const Tile32 &tm, int t, const float2 *__restrict__ x,
                                        HaloTile<float2> &xT, HaloTile<float2> &nT, int &k, float2 &y) {
  const GridDev &g = F.g;
  const int i0 = (t / tm.tiles_j) * TILE_I, j0 = (t % tm.tiles_j) * TILE_J;
  const int ti = threadIdx.x >> 5, tj = threadIdx.x & 31, i = i0 + ti, j = j0 + tj;
  const bool inside = i < g.Mx && j < g.My;
  k = inside ? i * g.My + j : 0;
  const uint32_t f = F.flags[k];
  const float bta = F.beta[k];
  __syncthreads();
  load_halo_tile<float2>(xT, i0, j0, g.Mx, g.My, [&](int ii, int jj) { return x[ii * g.My + jj]; });
  load_halo_tile<float2>(nT, i0, j0, g.Mx, g.My, [&](int ii, int jj) { return F.nuH[ii * g.My + jj]; });
  __syncthreads();
  if (!inside) return false;
  y = fine_apply_tile(F, i, j, f, bta, xT, nT, ti, tj);
  return true;
}

// start of an inner solve with d0 = 0: r = rhat = rhs, p = v = d = 0.  The outer test
// ||b - A x|| <= outer_rtol ||b|| and the inner tolerance (what this refinement step still
// needs, with a margin, never below inner_min) come from the FP64 norms in res2.
// DEV_RTOL: the outer tolerance is read from outer_rtol_dev (a whole-solve graph, whose
// tolerance changes from one Picard iteration to the next) instead of outer_rtol.
template <bool DEV_RTOL>
__global__ void __launch_bounds__(NT32) k32_init(int N, const float2 *__restrict__ rhs, float2 *__restrict__ r,
                                                 float2 *__restrict__ rhat, float2 *__restrict__ p,
                                                 float2 *__restrict__ v, float2 *__restrict__ d, double *partials,
                                                 unsigned *ticket, KState *st, const double *res2,
                                                 double outer_rtol, const double *outer_rtol_dev, double inner_min,
                                                 int maxit) {
  if constexpr (DEV_RTOL) outer_rtol = *outer_rtol_dev;
  const double rn = sqrt(res2[0]), bn = sqrt(res2[1]);
  const bool outer_done = !(rn > outer_rtol * bn) || bn == 0.0;   // NaN counts as done: the host reports it
  double acc[1] = {0.0};
  if (!outer_done)
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
      const float2 b = rhs[k], z = make_float2(0.0f, 0.0f);
      r[k] = b;
      rhat[k] = b;
      p[k] = z;
      v[k] = z;
      d[k] = z;
      acc[0] += dotf(b, b);
    }
  double tot[1];
  if (grid_reduce<1>(acc, partials, ticket, tot)) {
    st->outer_r2 = res2[0];
    st->outer_b2 = res2[1];
    st->rtol = fmin(0.5, fmax(inner_min, 0.7 * outer_rtol * bn / rn));
    st->maxit = maxit;
    st->rnorm2 = tot[0];
    st->bnorm2 = tot[0];
    st->rnorm0 = sqrt(tot[0]);
    st->rho = tot[0];
    st->alpha = 1.0;
    st->omega = 1.0;
    st->beta = 0.0;
    st->iter = 0;
    st->status = 0;
    st->done = (tot[0] == 0.0) ? 1 : 0;
    if (outer_done) {
      st->done = 1;
      st->status = KSP_OUTER_DONE;
    } else if (!isfinite(tot[0])) {
      st->done = 1;
      st->status = KSP_NAN;
    }
  }
}

__global__ void __launch_bounds__(NT32) k32_p(int N, const float2 *__restrict__ r, const float2 *__restrict__ v,
                                              float2 *__restrict__ p, const KState *st) {
  if (st->done) return;
  const float bta = (float)st->beta, om = (float)st->omega;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const float2 rk = r[k], pk = p[k], vk = v[k];
    p[k] = make_float2(rk.x + bta * (pk.x - om * vk.x), rk.y + bta * (pk.y - om * vk.y));
  }
}

// The tile loop of the two FP32 apply kernels: tiles whose rows can be staged by the bulk-copy
// engine go through two shared-memory stages (the next tile's rows in flight while this one
// computes); the rest (the first and last tile columns) load as before.  body(k, y) gets each
// cell's y = A x.  The same tiles in the same order per block as the plain loop, so the same
// sums.  A stage whose bounded wait gives up is computed from global memory instead, staging
// stops for the rest of the block's tiles, and the late copies are waited for (bounded) before
// the block exits; the return value then tells the caller to stop the solve.
template <class BODY>
__device__ __forceinline__ bool tile_loop_staged(const FineF &F, const Tile32 &tm, const float2 *__restrict__ x,
                                                 const BODY &body) {
  __shared__ HaloTile<float2> xT, nT;
  __shared__ TmaStage stg[2];
  __shared__ unsigned long long bars[2];
  if (threadIdx.x == 0) {
    tma_bar_init(&bars[0]);
    tma_bar_init(&bars[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int My = F.g.My;
  // block-uniform state: the phase parity of each stage's mbarrier (bit q for stage q);
  // stages whose copies came late (never reused); staging on; the current tile's rows were
  // issued into stage s
  unsigned parity = 0u, lost = 0u;
  bool staging = true, cur = false;
  int t = blockIdx.x, s = 0;
  if (t < tm.tiles) {
    const int i0 = (t / tm.tiles_j) * TILE_I, j0 = (t % tm.tiles_j) * TILE_J;
    if (tma_tile_ok(j0, My)) {
      tma_issue(stg[0], &bars[0], x, F, i0, j0);
      cur = true;
    }
  }
  __syncthreads();   // the first staged tile's offsets
  for (; t < tm.tiles; t += gridDim.x, s ^= 1) {
    const int tn = t + gridDim.x;
    bool next = false;
    if (staging && tn < tm.tiles) {
      const int i0n = (tn / tm.tiles_j) * TILE_I, j0n = (tn % tm.tiles_j) * TILE_J;
      if (tma_tile_ok(j0n, My)) {
        tma_issue(stg[s ^ 1], &bars[s ^ 1], x, F, i0n, j0n);
        next = true;
      }
    }
    const int i0 = (t / tm.tiles_j) * TILE_I, j0 = (t % tm.tiles_j) * TILE_J;
    int k = 0;
    float2 y;
    bool inside, late = false;
    if (cur) {
      late = !tma_wait(&bars[s], (parity >> s) & 1u);
      inside = late ? tma_apply_direct(F, x, i0, j0, k, y) : tma_apply(F, stg[s], i0, j0, k, y);
    } else {
      inside = apply32(F, tm, t, x, xT, nT, k, y);
    }
    if (inside) body(k, y);
    // stage s is free again (and the next staged tile's offsets are visible) unless late
    if (__syncthreads_or(late)) {
      staging = false;
      lost |= 1u << s;
    } else if (cur) {
      parity ^= 1u << s;
    }
    cur = next;
  }
  for (int q = 0; q < 2; ++q)
    if ((lost >> q) & 1u) tma_wait(&bars[q], (parity >> q) & 1u);
  return lost != 0u;
}

// y = A x over the tiles with the BiCGStab epilogue e (EpiV: v = A phat; EpiT: t = A shat);
// STAGED: interior tiles through the bulk-copy stages, else every tile by plain loads
template <class EPI, bool STAGED>
__global__ void __launch_bounds__(NT32) k32_apply(FineF F, Tile32 tm, const float2 *__restrict__ x, EPI e) {
  if (e.st->done) return;
  e.begin();
  auto body = [&](int k, const float2 &y) { e.body(k, y); };
  if constexpr (STAGED) {
    if (tile_loop_staged(F, tm, x, body) && threadIdx.x == 0) {
      e.st->done = 1;
      e.st->status = KSP_STALLED;
    }
  } else {
    __shared__ HaloTile<float2> xT, nT;
    for (int t = blockIdx.x; t < tm.tiles; t += gridDim.x) {
      int k = 0;
      float2 y;
      if (apply32(F, tm, t, x, xT, nT, k, y)) body(k, y);
    }
  }
  e.finish();
}

// d += alpha phat + omega shat; r = s - omega t with s = r - alpha v formed here
__global__ void __launch_bounds__(NT32) k32_x(int N, const float2 *__restrict__ phat, const float2 *__restrict__ shat,
                                              const float2 *__restrict__ v, const float2 *__restrict__ tv,
                                              const float2 *__restrict__ rhat, float2 *__restrict__ d,
                                              float2 *__restrict__ r, double *partials, unsigned *ticket,
                                              KState *st) {
  if (st->done) return;
  const float al = (float)st->alpha, om = (float)st->omega;
  double acc[2] = {0.0, 0.0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const float2 rk0 = r[k], vk = v[k];
    const float2 sk = make_float2(rk0.x - al * vk.x, rk0.y - al * vk.y);
    const float2 ph = phat[k], sh = shat[k], tk = tv[k];
    float2 dk = d[k];
    dk.x += al * ph.x + om * sh.x;
    dk.y += al * ph.y + om * sh.y;
    d[k] = dk;
    const float2 rk = make_float2(sk.x - om * tk.x, sk.y - om * tk.y);
    r[k] = rk;
    acc[0] += dotf(rhat[k], rk);
    acc[1] += dotf(rk, rk);
  }
  double tot[2];
  if (grid_reduce<2>(acc, partials, ticket, tot)) {
    const double rho_new = tot[0];
    st->rnorm2 = tot[1];
    st->iter += 1;
    const double rn = sqrt(tot[1]), tol = st->rtol * sqrt(st->bnorm2);
    if (!isfinite(rn)) {
      st->done = 1; st->status = KSP_NAN;
    } else if (rn <= tol) {
      st->done = 1; st->status = 0;
    } else if (st->iter >= st->maxit) {
      st->done = 1; st->status = KSP_MAXIT;
    } else if (om == 0.0f || rho_new == 0.0) {
      st->done = 1; st->status = KSP_BREAKDOWN;
    } else {
      st->beta = (rho_new / st->rho) * ((double)al / (double)om);
      st->rho = rho_new;
    }
  }
}

int blocks_n(const Launch &L, int n) { return std::min((n + NT32 - 1) / NT32, L.max_blocks); }

}  // namespace

void launch_mixed_init(const Launch &L, int N, const Krylov32 &K, const double *res2, double outer_rtol,
                       double inner_min, int maxit) {
  k32_init<false><<<blocks_n(L, N), NT32, 0, L.stream>>>(N, K.rhs, K.r, K.rhat, K.p, K.v, K.d, L.partials, L.ticket,
                                                         K.st, res2, outer_rtol, nullptr, inner_min, maxit);
  L.tick();
}

void launch_mixed_init_dev(const Launch &L, int N, const Krylov32 &K, const double *res2, const double *outer_rtol,
                           double inner_min, int maxit) {
  k32_init<true><<<blocks_n(L, N), NT32, 0, L.stream>>>(N, K.rhs, K.r, K.rhat, K.p, K.v, K.d, L.partials, L.ticket,
                                                        K.st, res2, 0.0, outer_rtol, inner_min, maxit);
  L.tick();
}

void launch_mixed_iteration(const Launch &L, const GridDev &g, const Fields &f, const MGHierarchy &H,
                            const Krylov32 &K) {
  const int N = g.Mx * g.My;
  const FineF F = fine_view(g, f, H);
  const Tile32 tm = tiles32(g);
  const int bv = blocks_n(L, N), bt = std::min(tm.tiles, L.max_blocks);
  const EpiV ev{K.rhat, K.v, L.partials, L.ticket, K.st, {0.0}};
  const EpiT et{K.r, K.v, K.t, L.partials, L.ticket, K.st, {0.0, 0.0}, 0.0f};
  k32_p<<<bv, NT32, 0, L.stream>>>(N, K.r, K.v, K.p, K.st);
  if (H.apply_kernel == 2) {   // the V-cycles' fine-level passes apply A to their results
    mg_vcycle_apply(L, g, f, H, K.p, K.phat, ev);
    mg_vcycle_s_apply(L, g, f, H, K.r, K.v, K.shat, et);   // s = r - alpha v is not stored
  } else {
    const bool staged = H.apply_kernel == 1;
    mg_vcycle(L, g, f, H, K.p, K.phat, K.st);
    if (staged) k32_apply<EpiV, true><<<bt, NT32, 0, L.stream>>>(F, tm, K.phat, ev);
    else k32_apply<EpiV, false><<<bt, NT32, 0, L.stream>>>(F, tm, K.phat, ev);
    mg_vcycle_s(L, g, f, H, K.r, K.v, K.shat, K.st);   // s = r - alpha v is not stored
    if (staged) k32_apply<EpiT, true><<<bt, NT32, 0, L.stream>>>(F, tm, K.shat, et);
    else k32_apply<EpiT, false><<<bt, NT32, 0, L.stream>>>(F, tm, K.shat, et);
    L.tick(2);
  }
  k32_x<<<bv, NT32, 0, L.stream>>>(N, K.phat, K.shat, K.v, K.t, K.rhat, K.d, K.r, L.partials, L.ticket, K.st);
  L.tick(2);
}

}  // namespace pism_gpu
