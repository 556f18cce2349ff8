// ssa_tma_tile.cuh — halo tiles of the FP32 fine-level fields staged by the bulk-copy engine
// (TMA, cp.async.bulk), double-buffered: while a block computes one 32 x 8 tile, the rows of
// its next tile are in flight.
//
// A tile's halo rows (34 cells of x and of nu*H, j0 - 1 .. j0 + 32) and own rows (32 cells of
// the flag word and of beta) are contiguous in memory but do not start on 16-byte
// boundaries (801-cell rows); each staged row therefore copies 36 cells from the 16-byte
// boundary at or before its first cell and keeps that offset.  The rows of every array wrap
// periodically in i by their address; tiles whose columns would wrap in j (the first and the
// last tile column or two) take the plain load path instead.
#pragma once

#include "ssa_fine32.cuh"

namespace pism_gpu {

constexpr int TMA_ROW = TILE_J + 4;   // cells per staged row

struct __align__(16) TmaStage {
  float2 x[TILE_I + 2][TMA_ROW];   // halo rows of the vector the stencil is applied to
  float2 n[TILE_I + 2][TMA_ROW];   // halo rows of FP32 nu*H
  uint32_t f[TILE_I][TMA_ROW];     // own rows of the flag word
  float b[TILE_I][TMA_ROW];        // own rows of FP32 beta
  int ox[TILE_I + 2];              // offset of column j0 - 1 in each staged x / n row
  int of[TILE_I];                  // offset of column j0 in each staged f / b row
};
static_assert(sizeof(float2) * (TILE_I + 2) * TMA_ROW % 16 == 0 && sizeof(float) * TILE_I * TMA_ROW % 16 == 0,
              "staged rows keep every array 16-byte aligned");

// whether a tile starting at column j0 takes the staged path: no row segment wraps in j and
// every rounded-out segment stays inside its array
__device__ __forceinline__ bool tma_tile_ok(int j0, int My) { return j0 >= TILE_J && j0 + TMA_ROW <= My; }

__device__ __forceinline__ unsigned tma_smem(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_bar_init(unsigned long long *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tma_smem(bar)) : "memory");
}

__device__ __forceinline__ void tma_copy(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tma_smem(dst)),
               "l"(src), "r"(bytes), "r"(tma_smem(bar))
               : "memory");
}

// bounded wait for the phase `parity` of a stage's mbarrier; false when it did not complete
__device__ __forceinline__ bool tma_wait(unsigned long long *bar, unsigned parity) {
  const unsigned a = tma_smem(bar);
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Warp 0 stages tile (i0, j0) (tma_tile_ok) into S: lane 0 announces the bytes on the
// mbarrier, then the lanes issue one bulk copy per staged row (10 rows of x and of nu*H, the
// tile's rows inside the grid of the flags and of beta).  The offsets are plain stores; the
// caller orders them before their readers with a __syncthreads.
__device__ __forceinline__ void tma_issue(TmaStage &S, unsigned long long *bar, const float2 *__restrict__ x,
                                          const FineF &F, int i0, int j0) {
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x, Mx = F.g.Mx, My = F.g.My;
  const int own = Mx - i0 < TILE_I ? Mx - i0 : TILE_I;
  if (lane == 0) {
    const unsigned bytes = 2u * (TILE_I + 2) * TMA_ROW * sizeof(float2) + 2u * own * TMA_ROW * sizeof(float);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tma_smem(bar)), "r"(bytes)
                 : "memory");
  }
  __syncwarp();
  for (int q = lane; q < 2 * (TILE_I + 2) + 2 * own; q += 32) {
    if (q < 2 * (TILE_I + 2)) {
      const int a = q % (TILE_I + 2);
      const int ii = pmod(i0 - 1 + a, Mx);
      const long long e = (long long)ii * My + j0 - 1, ea = e & ~1LL;   // 16-byte boundary of float2
      if (q < TILE_I + 2) {
        S.ox[a] = (int)(e - ea);
        tma_copy(&S.x[a][0], x + ea, TMA_ROW * sizeof(float2), bar);
      } else {
        tma_copy(&S.n[a][0], F.nuH + ea, TMA_ROW * sizeof(float2), bar);
      }
    } else {
      const int r = q - 2 * (TILE_I + 2), a = r % own;
      const long long e = (long long)(i0 + a) * My + j0, ea = e & ~3LL;   // 16-byte boundary of 4-byte cells
      if (r < own) {
        S.of[a] = (int)(e - ea);
        tma_copy(&S.f[a][0], F.flags + ea, TMA_ROW * sizeof(uint32_t), bar);
      } else {
        tma_copy(&S.b[a][0], F.beta + ea, TMA_ROW * sizeof(float), bar);
      }
    }
  }
}

// y = A x at this thread's cell of a staged tile; false outside the grid
__device__ __forceinline__ bool tma_apply(const FineF &F, const TmaStage &S, int i0, int j0, int &k, float2 &y) {
  const int ti = threadIdx.x >> 5, tj = threadIdx.x & 31, i = i0 + ti, j = j0 + tj;
  if (i >= F.g.Mx) return false;   // j < My on a staged tile
  k = i * F.g.My + j;
  const int o = S.of[ti];
  const uint32_t f = S.f[ti][tj + o];
  const float bta = S.b[ti][tj + o];
  auto xr = [&](int di, int dj) { return S.x[ti + 1 + di][tj + 1 + dj + S.ox[ti + 1 + di]]; };
  const int om = S.ox[ti], oc = S.ox[ti + 1];
  y = fine_apply_coef(F, i, j, f, bta, S.n[ti][tj + 1 + om].x, S.n[ti + 1][tj + 1 + oc].x, S.n[ti + 1][tj + oc].y,
                      S.n[ti + 1][tj + 1 + oc].y, xr);
  return true;
}

// y = A x at this thread's cell of a tile that could be staged (tma_tile_ok), read straight
// from global memory: for a staged tile whose copies did not arrive in time.  The same
// operands as tma_apply, so the same bits.
__device__ __forceinline__ bool tma_apply_direct(const FineF &F, const float2 *__restrict__ x, int i0, int j0, int &k,
                                                 float2 &y) {
  const int Mx = F.g.Mx, My = F.g.My, i = i0 + (threadIdx.x >> 5), j = j0 + (threadIdx.x & 31);
  if (i >= Mx) return false;
  k = i * My + j;
  const int rm = pmod(i - 1, Mx) * My + j, rp = pmod(i + 1, Mx) * My + j;
  auto xr = [&](int di, int dj) { return x[(di < 0 ? rm : di > 0 ? rp : k) + dj]; };
  y = fine_apply_coef(F, i, j, F.flags[k], F.beta[k], F.nuH[rm].x, F.nuH[k].x, F.nuH[k - 1].y, F.nuH[k].y, xr);
  return true;
}

}  // namespace pism_gpu
