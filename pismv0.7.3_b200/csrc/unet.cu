// unet.cu — the learned warm start's network (include/pism_unet_gpu.h): a 4-level U-Net in
// BF16 with FP32 accumulation on the tensor cores (mma.sync m16n8k16, operands staged in
// shared memory and fed by ldmatrix), its backward pass and an Adam step.
//
// The convolutions are implicit GEMMs over an 8 x 16 pixel output tile: the CTA stages the
// 10 x 18 input patch of one 16- or 32-channel slice and the 3 x 3 x 32 weights of its 32
// output channels, each warp owns one output row (M = 16 pixels) and all 32 channels
// (4 n-blocks of 8), K runs over taps x channels.  The backward data pass is the same kernel
// on flipped, transposed weights with the ReLU mask applied while staging; the weight
// gradient is a GEMM over pixels (one warp per tap) reduced deterministically across CTAs.
// Every reduction (weight / bias gradients, loss) is written as per-CTA partial sums and
// summed in a fixed order, so training runs are bit-reproducible.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "pism_unet_gpu.h"
#include "unet_internal.h"

using bf16 = __nv_bfloat16;

namespace pism_unet {

constexpr int TH = 8, TW = 16;            // output tile
constexpr int PH = TH + 2, PW = TW + 2;   // input patch with the 3 x 3 halo
constexpr int NT = 32;                    // output channels per CTA
constexpr int THREADS = 256;              // 8 warps = 8 tile rows
constexpr int WG_THREADS = 288;           // weight gradient: 9 warps = 9 taps
constexpr int WG_MAX_CTAS = 64;           // pixel-range partial sums per weight gradient

// ---- the network ----
struct LayerDef {
  int cin, cout, level;   // level 0 = full resolution
};
constexpr int NLAYERS = 10;
constexpr LayerDef LAYERS[NLAYERS] = {
    {16, 32, 0}, {32, 32, 0}, {32, 64, 1}, {64, 64, 1}, {64, 96, 2},
    {96, 96, 2}, {96, 128, 3}, {224, 96, 2}, {160, 64, 1}, {96, 32, 0},
};
constexpr int HEAD_CIN = 32, HEAD_COUT = 2;

long long param_count() {
  long long n = 0;
  for (const LayerDef &L : LAYERS) n += 9LL * L.cout * L.cin + L.cout;
  return n + HEAD_COUT * HEAD_CIN + HEAD_COUT;
}

// ---- device helpers ----
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void *p) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void *p) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

// d += a (16x16, row) * b (16x8, col), BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// keep the BF16 halves of v whose counterpart in m is > 0 (the ReLU derivative)
__device__ __forceinline__ uint32_t relu_mask2(uint32_t v, uint32_t m) {
  uint32_t keep = 0;
  if (!(m & 0x8000u) && (m & 0x7fffu)) keep |= 0x0000ffffu;
  if (!(m & 0x80000000u) && (m & 0x7fff0000u)) keep |= 0xffff0000u;
  return v & keep;
}

__device__ __forceinline__ uint4 relu_mask8(uint4 v, uint4 m) {
  return make_uint4(relu_mask2(v.x, m.x), relu_mask2(v.y, m.y), relu_mask2(v.z, m.z), relu_mask2(v.w, m.w));
}

__device__ __forceinline__ void unpack8(uint4 v, float (&f)[8]) {
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float2 t = __bfloat1622float2(h[q]);
    f[2 * q] = t.x;
    f[2 * q + 1] = t.y;
  }
}

__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint4 v;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&v);
#pragma unroll
  for (int q = 0; q < 4; ++q) h[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
  return v;
}

// Stage the (TH+2) x (TW+2) patch of channels [c0, c0 + CS) around the tile at (i0, j0) of
// image b; zero outside the image; masked by (mask > 0) when mask is given.
template <int CS, int NTHR>
__device__ __forceinline__ void stage_patch(bf16 *patch, const bf16 *__restrict__ x, const bf16 *__restrict__ mask,
                                            int C, int c0, int b, int i0, int j0, int H, int W) {
  constexpr int CP = CS + 8, CH = CS / 8;
  for (int q = threadIdx.x; q < PH * PW * CH; q += NTHR) {
    const int pix = q / CH, ch = q - pix * CH;
    const int pi = pix / PW, pj = pix - pi * PW;
    const int ii = i0 - 1 + pi, jj = j0 - 1 + pj;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (ii >= 0 && ii < H && jj >= 0 && jj < W) {
      const size_t off = (((size_t)b * H + ii) * W + jj) * C + c0 + ch * 8;
      v = *reinterpret_cast<const uint4 *>(x + off);
      if (mask) v = relu_mask8(v, *reinterpret_cast<const uint4 *>(mask + off));
    }
    *reinterpret_cast<uint4 *>(patch + pix * CP + ch * 8) = v;
  }
}

// ---- 3x3 convolution (forward, and backward data on flipped weights) ----
// y[b, i, j, co] = act(bias[co] + sum_{tap, ci} w[tap, co, ci] * xm[b, i + ky - 1, j + kx - 1, ci])
// xm = x * (mask > 0) when mask is given.  grid = (B * tiles, Cout / 32).
template <int CS>
__global__ void __launch_bounds__(THREADS) k_conv3x3(const bf16 *__restrict__ x, const bf16 *__restrict__ xmask,
                                                     int Cin, const bf16 *__restrict__ w,
                                                     const float *__restrict__ bias, int relu, bf16 *__restrict__ y,
                                                     int Cout, int H, int W) {
  constexpr int CP = CS + 8, CH = CS / 8;
  __shared__ __align__(16) bf16 patch[PH * PW * CP];
  __shared__ __align__(16) bf16 wsm[9 * NT * CP];
  const int tiles_w = (W + TW - 1) / TW, tiles_h = (H + TH - 1) / TH;
  int t = blockIdx.x;
  const int b = t / (tiles_h * tiles_w);
  t -= b * tiles_h * tiles_w;
  const int i0 = (t / tiles_w) * TH, j0 = (t % tiles_w) * TW;
  const int co0 = blockIdx.y * NT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // ldmatrix row addresses: A (pixels x channels, row-major), B (channels x couts, stored [cout][cin])
  const int am = (lane & 7) + 8 * ((lane >> 3) & 1), ak = 8 * (lane >> 4);
  const int bn = (lane & 7) + 8 * (lane >> 4), bk = 8 * ((lane >> 3) & 1);
  float acc[NT / 8][4];
#pragma unroll
  for (int n = 0; n < NT / 8; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.0f;
  for (int c0 = 0; c0 < Cin; c0 += CS) {
    stage_patch<CS, THREADS>(patch, x, xmask, Cin, c0, b, i0, j0, H, W);
    for (int q = threadIdx.x; q < 9 * NT * CH; q += THREADS) {
      const int row = q / CH, ch = q - row * CH;   // row = tap * NT + n
      const int tap = row / NT, n = row - tap * NT;
      *reinterpret_cast<uint4 *>(wsm + row * CP + ch * 8) =
          *reinterpret_cast<const uint4 *>(w + ((size_t)tap * Cout + co0 + n) * Cin + c0 + ch * 8);
    }
    __syncthreads();
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int ky = tap / 3, kx = tap - 3 * (tap / 3);
#pragma unroll
      for (int kk = 0; kk < CS; kk += 16) {
        uint32_t a[4];
        ldsm_x4(a, patch + ((warp + ky) * PW + am + kx) * CP + kk + ak);
#pragma unroll
        for (int nb2 = 0; nb2 < NT / 16; ++nb2) {
          uint32_t bb[4];
          ldsm_x4(bb, wsm + (tap * NT + nb2 * 16 + bn) * CP + kk + bk);
          mma_bf16(acc[2 * nb2], a, bb[0], bb[1]);
          mma_bf16(acc[2 * nb2 + 1], a, bb[2], bb[3]);
        }
      }
    }
    __syncthreads();
  }
  const int g = lane >> 2, tq = lane & 3, i = i0 + warp;
  if (i >= H) return;
#pragma unroll
  for (int nb = 0; nb < NT / 8; ++nb) {
    const int co = co0 + nb * 8 + 2 * tq;
    const float b0 = bias ? bias[co] : 0.0f, b1 = bias ? bias[co + 1] : 0.0f;
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const int j = j0 + g + 8 * hh;
      if (j >= W) continue;
      float v0 = acc[nb][2 * hh] + b0, v1 = acc[nb][2 * hh + 1] + b1;
      if (relu) {
        v0 = fmaxf(v0, 0.0f);
        v1 = fmaxf(v1, 0.0f);
      }
      *reinterpret_cast<__nv_bfloat162 *>(y + (((size_t)b * H + i) * W + j) * Cout + co) =
          __floats2bfloat162_rn(v0, v1);
    }
  }
}

// ---- weight gradient ----
// part[cta][tap][co][ci] = sum over the CTA's pixel tiles of dym[p, co] * x[p + tap offset, ci],
// dym = dy * (ymask > 0).  grid = (ctas over pixel tiles, (Cout / 32) * (Cin / CS)).
template <int CS>
__global__ void __launch_bounds__(WG_THREADS) k_conv3x3_wgrad(const bf16 *__restrict__ x, int Cin,
                                                              const bf16 *__restrict__ dy,
                                                              const bf16 *__restrict__ ymask, int Cout, int B, int H,
                                                              int W, float *__restrict__ part) {
  constexpr int CP = CS + 8, DP = NT + 8;
  __shared__ __align__(16) bf16 patch[PH * PW * CP];
  __shared__ __align__(16) bf16 dys[TH * TW * DP];
  const int nci = Cin / CS;
  const int co0 = (blockIdx.y / nci) * NT, ci0 = (blockIdx.y % nci) * CS;
  const int tiles_w = (W + TW - 1) / TW, tiles_h = (H + TH - 1) / TH, tiles = B * tiles_h * tiles_w;
  const int tap = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ky = tap / 3, kx = tap - 3 * (tap / 3);
  // A = dy^T (couts x pixels) from [pixel][cout]; B = x (pixels x cins) from [pixel][cin]
  const int apx = (lane & 7) + 8 * (lane >> 4), amo = 8 * ((lane >> 3) & 1);
  const int bpx = (lane & 7) + 8 * ((lane >> 3) & 1), bno = 8 * (lane >> 4);
  float acc[2][CS / 8][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int n = 0; n < CS / 8; ++n) acc[m][n][0] = acc[m][n][1] = acc[m][n][2] = acc[m][n][3] = 0.0f;
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    int r = t;
    const int b = r / (tiles_h * tiles_w);
    r -= b * tiles_h * tiles_w;
    const int i0 = (r / tiles_w) * TH, j0 = (r % tiles_w) * TW;
    stage_patch<CS, WG_THREADS>(patch, x, nullptr, Cin, ci0, b, i0, j0, H, W);
    for (int q = threadIdx.x; q < TH * TW * (NT / 8); q += WG_THREADS) {
      const int pix = q / (NT / 8), ch = q - pix * (NT / 8);
      const int ii = i0 + pix / TW, jj = j0 + pix % TW;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (ii < H && jj < W) {
        const size_t off = (((size_t)b * H + ii) * W + jj) * Cout + co0 + ch * 8;
        v = *reinterpret_cast<const uint4 *>(dy + off);
        if (ymask) v = relu_mask8(v, *reinterpret_cast<const uint4 *>(ymask + off));
      }
      *reinterpret_cast<uint4 *>(dys + pix * DP + ch * 8) = v;
    }
    __syncthreads();
#pragma unroll 2
    for (int row = 0; row < TH; ++row) {
      uint32_t a[2][4];
#pragma unroll
      for (int mb = 0; mb < 2; ++mb) ldsm_x4_t(a[mb], dys + (row * TW + apx) * DP + mb * 16 + amo);
#pragma unroll
      for (int nb2 = 0; nb2 < CS / 16; ++nb2) {
        uint32_t bb[4];
        ldsm_x4_t(bb, patch + ((row + ky) * PW + bpx + kx) * CP + nb2 * 16 + bno);
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
          mma_bf16(acc[mb][2 * nb2], a[mb], bb[0], bb[1]);
          mma_bf16(acc[mb][2 * nb2 + 1], a[mb], bb[2], bb[3]);
        }
      }
    }
    __syncthreads();
  }
  const int g = lane >> 2, tq = lane & 3;
  float *dst = part + ((size_t)blockIdx.x * 9 + tap) * Cout * Cin;
#pragma unroll
  for (int mb = 0; mb < 2; ++mb)
#pragma unroll
    for (int nb = 0; nb < CS / 8; ++nb)
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int co = co0 + mb * 16 + g + 8 * hh, ci = ci0 + nb * 8 + 2 * tq;
        *reinterpret_cast<float2 *>(dst + (size_t)co * Cin + ci) = make_float2(acc[mb][nb][2 * hh], acc[mb][nb][2 * hh + 1]);
      }
}

// out[k] = sum_{s < nparts} part[s * n + k], in order
__global__ void k_reduce_parts(const float *__restrict__ part, int nparts, int n, float *__restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int q = 0; q < nparts; ++q) s += part[(size_t)q * n + k];
    out[k] = s;
  }
}

// part[cta][c] = sum over the CTA's pixels of dy[p, c] * (ymask[p, c] > 0)
__global__ void __launch_bounds__(256) k_bias_grad(const bf16 *__restrict__ dy, const bf16 *__restrict__ ymask, int C,
                                                   long long P, float *__restrict__ part) {
  __shared__ float red[256];
  const int lanes = 256 / C;   // pixels in flight per CTA
  const int c = threadIdx.x % C, l = threadIdx.x / C;
  float s = 0.0f;
  if (l < lanes) {
    for (long long p = (long long)blockIdx.x * lanes + l; p < P; p += (long long)gridDim.x * lanes) {
      const bf16 v = dy[p * C + c];
      const bf16 m = ymask[p * C + c];
      if (__bfloat162float(m) > 0.0f) s += __bfloat162float(v);
    }
  }
  red[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < C) {
    float t = 0.0f;
    for (int q = 0; q < lanes; ++q) t += red[q * C + threadIdx.x];
    part[(size_t)blockIdx.x * C + threadIdx.x] = t;
  }
}

// wt[8 - tap][ci][co] = w[tap][co][ci]: the backward-data weights
__global__ void k_flip_weights(const bf16 *__restrict__ w, int Cout, int Cin, bf16 *__restrict__ wt) {
  const int n = 9 * Cout * Cin;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int tap = k / (Cout * Cin), r = k - tap * Cout * Cin, co = r / Cin, ci = r - co * Cin;
    wt[((size_t)(8 - tap) * Cin + ci) * Cout + co] = w[k];
  }
}

// ---- pooling, upsampling + concatenation ----
// y[b, I, J, :] = mean of x over the 2 x 2 block; 8 channels per thread
__global__ void k_pool(const bf16 *__restrict__ x, int C, int B, int H, int W, bf16 *__restrict__ y) {
  const int h = H / 2, w = W / 2, CH = C / 8;
  const long long n = (long long)B * h * w * CH;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(k % CH);
    long long p = k / CH;
    const int J = (int)(p % w);
    p /= w;
    const int I = (int)(p % h);
    const int b = (int)(p / h);
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      float f[8];
      unpack8(*reinterpret_cast<const uint4 *>(x + (((size_t)b * H + 2 * I + (d >> 1)) * W + 2 * J + (d & 1)) * C + ch * 8), f);
#pragma unroll
      for (int q = 0; q < 8; ++q) s[q] += f[q];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) s[q] *= 0.25f;
    *reinterpret_cast<uint4 *>(y + (((size_t)b * h + I) * w + J) * C + ch * 8) = pack8(s);
  }
}

// dx[b, i, j, :] += dy[b, i/2, j/2, :] / 4
__global__ void k_pool_back_add(const bf16 *__restrict__ dy, int C, int B, int H, int W, bf16 *__restrict__ dx) {
  const int h = H / 2, w = W / 2, CH = C / 8;
  const long long n = (long long)B * H * W * CH;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(k % CH);
    long long p = k / CH;
    const int j = (int)(p % W);
    p /= W;
    const int i = (int)(p % H);
    const int b = (int)(p / H);
    float a[8], d[8];
    bf16 *dst = dx + (((size_t)b * H + i) * W + j) * C + ch * 8;
    unpack8(*reinterpret_cast<const uint4 *>(dst), a);
    unpack8(*reinterpret_cast<const uint4 *>(dy + (((size_t)b * h + i / 2) * w + j / 2) * C + ch * 8), d);
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] += 0.25f * d[q];
    *reinterpret_cast<uint4 *>(dst) = pack8(a);
  }
}

// c[b, i, j, :] = [u[b, i/2, j/2, 0:Cu], s[b, i, j, 0:Cs]]
__global__ void k_upcat(const bf16 *__restrict__ u, int Cu, const bf16 *__restrict__ s, int Cs, int B, int H, int W,
                        bf16 *__restrict__ c) {
  const int C = Cu + Cs, CH = C / 8, h = H / 2, w = W / 2;
  const long long n = (long long)B * H * W * CH;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(k % CH);
    long long p = k / CH;
    const int j = (int)(p % W);
    p /= W;
    const int i = (int)(p % H);
    const int b = (int)(p / H);
    const int c0 = ch * 8;
    const uint4 v = c0 < Cu ? *reinterpret_cast<const uint4 *>(u + (((size_t)b * h + i / 2) * w + j / 2) * Cu + c0)
                            : *reinterpret_cast<const uint4 *>(s + (((size_t)b * H + i) * W + j) * Cs + c0 - Cu);
    *reinterpret_cast<uint4 *>(c + (((size_t)b * H + i) * W + j) * C + c0) = v;
  }
}

// du[b, I, J, :] = sum of dc[b, 2I + di, 2J + dj, 0:Cu];  ds[b, i, j, :] = dc[b, i, j, Cu:]
__global__ void k_upcat_back(const bf16 *__restrict__ dc, int Cu, int Cs, int B, int H, int W, bf16 *__restrict__ du,
                             bf16 *__restrict__ ds) {
  const int C = Cu + Cs, h = H / 2, w = W / 2;
  const long long nu = (long long)B * h * w * (Cu / 8), ns = (long long)B * H * W * (Cs / 8);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nu + ns;
       k += (long long)gridDim.x * blockDim.x) {
    if (k < nu) {
      const int CH = Cu / 8, ch = (int)(k % CH);
      long long p = k / CH;
      const int J = (int)(p % w);
      p /= w;
      const int I = (int)(p % h);
      const int b = (int)(p / h);
      float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        float f[8];
        unpack8(*reinterpret_cast<const uint4 *>(dc + (((size_t)b * H + 2 * I + (d >> 1)) * W + 2 * J + (d & 1)) * C + ch * 8), f);
#pragma unroll
        for (int q = 0; q < 8; ++q) s[q] += f[q];
      }
      *reinterpret_cast<uint4 *>(du + (((size_t)b * h + I) * w + J) * Cu + ch * 8) = pack8(s);
    } else {
      const long long kk = k - nu;
      const int CH = Cs / 8, ch = (int)(kk % CH);
      const long long p = kk / CH;
      *reinterpret_cast<uint4 *>(ds + p * Cs + ch * 8) = *reinterpret_cast<const uint4 *>(dc + p * C + Cu + ch * 8);
    }
  }
}

// ---- input packing, head, loss ----
// x16[p, 0:8] = bf16(in[p, 0:8]), x16[p, 8:16] = 0
__global__ void k_pack_input(const float *__restrict__ in, long long P, bf16 *__restrict__ x16) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    float f[8];
    const float4 a = reinterpret_cast<const float4 *>(in)[2 * p], b = reinterpret_cast<const float4 *>(in)[2 * p + 1];
    f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w;
    f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
    reinterpret_cast<uint4 *>(x16)[2 * p] = pack8(f);
    reinterpret_cast<uint4 *>(x16)[2 * p + 1] = make_uint4(0u, 0u, 0u, 0u);
  }
}

// y[p, o] = bh[o] + sum_c d1[p, c] * Wh[o, c]
__global__ void k_head(const bf16 *__restrict__ d1, const float *__restrict__ wh, long long P, float *__restrict__ y) {
  __shared__ float ws[HEAD_COUT * HEAD_CIN + HEAD_COUT];
  for (int q = threadIdx.x; q < HEAD_COUT * HEAD_CIN + HEAD_COUT; q += blockDim.x) ws[q] = wh[q];
  __syncthreads();
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    float y0 = ws[2 * HEAD_CIN], y1 = ws[2 * HEAD_CIN + 1];
#pragma unroll
    for (int ch = 0; ch < HEAD_CIN / 8; ++ch) {
      float f[8];
      unpack8(reinterpret_cast<const uint4 *>(d1 + p * HEAD_CIN)[ch], f);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        y0 = fmaf(f[q], ws[ch * 8 + q], y0);
        y1 = fmaf(f[q], ws[HEAD_CIN + ch * 8 + q], y1);
      }
    }
    reinterpret_cast<float2 *>(y)[p] = make_float2(y0, y1);
  }
}

// per CTA: {sum w (y - t)^2, sum w}
__global__ void __launch_bounds__(256) k_loss_parts(const float *__restrict__ y, const float *__restrict__ t,
                                                    const float *__restrict__ wgt, long long P, float *__restrict__ part) {
  __shared__ float r0[256], r1[256];
  float s0 = 0.0f, s1 = 0.0f;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const float w = wgt ? wgt[p] : 1.0f;
    const float2 a = reinterpret_cast<const float2 *>(y)[p], b = reinterpret_cast<const float2 *>(t)[p];
    s0 += w * ((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y));
    s1 += w;
  }
  r0[threadIdx.x] = s0;
  r1[threadIdx.x] = s1;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      r0[threadIdx.x] += r0[threadIdx.x + o];
      r1[threadIdx.x] += r1[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = r0[0];
    part[2 * blockIdx.x + 1] = r1[0];
  }
}

// sums = {ordered sum of the loss parts, sum of weights, loss = sums[0] / (2 sums[1])}
__global__ void k_loss_finish(const float *__restrict__ part, int nparts, float *__restrict__ sums) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float a = 0.0f, b = 0.0f;
    for (int q = 0; q < nparts; ++q) {
      a += part[2 * q];
      b += part[2 * q + 1];
    }
    sums[0] = a;
    sums[1] = b;
    sums[2] = b > 0.0f ? a / (2.0f * b) : 0.0f;
  }
}

// dy = w (y - t) / sum w;  dd1[p, c] = sum_o dy[p, o] Wh[o, c];
// part[cta] = {dWh[2][32], dbh[2]} partial sums
__global__ void __launch_bounds__(256) k_head_back(const bf16 *__restrict__ d1, const float *__restrict__ y,
                                                   const float *__restrict__ t, const float *__restrict__ wgt,
                                                   const float *__restrict__ sums, const float *__restrict__ wh,
                                                   long long P, bf16 *__restrict__ dd1, float *__restrict__ part) {
  constexpr int NG = HEAD_COUT * HEAD_CIN + HEAD_COUT;
  __shared__ float red[NG][33];
  float g[NG];
#pragma unroll
  for (int q = 0; q < NG; ++q) g[q] = 0.0f;
  const float inv = sums[1] > 0.0f ? 1.0f / sums[1] : 0.0f;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const float w = (wgt ? wgt[p] : 1.0f) * inv;
    const float2 a = reinterpret_cast<const float2 *>(y)[p], b = reinterpret_cast<const float2 *>(t)[p];
    const float e0 = w * (a.x - b.x), e1 = w * (a.y - b.y);
#pragma unroll
    for (int ch = 0; ch < HEAD_CIN / 8; ++ch) {
      float f[8], o[8];
      unpack8(reinterpret_cast<const uint4 *>(d1 + p * HEAD_CIN)[ch], f);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int c = ch * 8 + q;
        o[q] = e0 * wh[c] + e1 * wh[HEAD_CIN + c];
        g[c] = fmaf(e0, f[q], g[c]);
        g[HEAD_CIN + c] = fmaf(e1, f[q], g[HEAD_CIN + c]);
      }
      reinterpret_cast<uint4 *>(dd1 + p * HEAD_CIN)[ch] = pack8(o);
    }
    g[2 * HEAD_CIN] += e0;
    g[2 * HEAD_CIN + 1] += e1;
  }
  // warp sums, then the 8 warps in order
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NG; ++q) {
    float v = g[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < NG) {
    float s = 0.0f;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[threadIdx.x][q];
    part[(size_t)blockIdx.x * NG + threadIdx.x] = s;
  }
}

// Adam with bias correction; the BF16 copy of every parameter follows the FP32 master
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2,
                       bf16 *__restrict__ p16) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.0f - b1) * gk;
    const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float pk = p[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    p[k] = pk;
    p16[k] = __float2bfloat16_rn(pk);
  }
}

__global__ void k_to_bf16(const float *__restrict__ p, long long n, bf16 *__restrict__ p16) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    p16[k] = __float2bfloat16_rn(p[k]);
}

// ---- the SSA side: features and the velocity from the network output ----
__global__ void k_features(int Mx, int My, int stride, const double *__restrict__ H, const double *__restrict__ bed,
                           const double *__restrict__ tauc, const double2 *__restrict__ hardness,
                           const int8_t *__restrict__ mask, const double2 *__restrict__ taud,
                           float *__restrict__ out, int height, int width) {
  const long long n = (long long)height * width;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int I = (int)(q / width), J = (int)(q % width);
    const int i = I * stride, j = J * stride;
    float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (i < Mx && j < My) {
      const size_t k = (size_t)i * My + j;
      const int m = mask[k];
      const double2 hb = hardness[k];
      const double hv = fmax(hb.x, hb.y);
      f[0] = (float)(H[k] * 1e-3);
      f[1] = (float)(bed[k] * 1e-3);
      f[2] = (float)log(fmax(tauc[k], 1.0) / 5.0e4);
      f[3] = (m == 2 || m == 3) && hv > 0.0 ? (float)(hv * 1e-8) : 0.0f;
      f[4] = m == 2 ? 1.0f : 0.0f;
      f[5] = m == 3 ? 1.0f : 0.0f;
      f[6] = (float)(taud[k].x * 1e-5);
      f[7] = (float)(taud[k].y * 1e-5);
    }
    float4 *o = reinterpret_cast<float4 *>(out + q * 8);
    o[0] = make_float4(f[0], f[1], f[2], f[3]);
    o[1] = make_float4(f[4], f[5], f[6], f[7]);
  }
}

// vel(i, j) = 10 m/yr * sinh(y) at the coarse points, bilinear in between (stride 1 or 2)
__global__ void k_velocity(const float *__restrict__ y, int height, int width, int stride, int Mx, int My,
                           double secpera, double2 *__restrict__ vel) {
  const long long n = (long long)Mx * My;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / My), j = (int)(k % My);
    const int I0 = i / stride, J0 = j / stride;
    const int I1 = min(I0 + (i % stride ? 1 : 0), height - 1), J1 = min(J0 + (j % stride ? 1 : 0), width - 1);
    double u = 0.0, v = 0.0;
    const int Is[2] = {I0, I1}, Js[2] = {J0, J1};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const float2 o = reinterpret_cast<const float2 *>(y)[(size_t)Is[a] * width + Js[b]];
        u += 10.0 * sinh((double)o.x);
        v += 10.0 * sinh((double)o.y);
      }
    vel[k] = make_double2(0.25 * u / secpera, 0.25 * v / secpera);
  }
}

// ---- the learned preconditioner correction: the residual's image and the correction ----
constexpr int PC_THREADS = 256;

// channels 6, 7 of the image = the stride x stride block means of s = D^-1 r (the
// block-Jacobi-scaled residual, in velocity units); per block the partial sum of their squares
__global__ void __launch_bounds__(PC_THREADS) k_pc_image(int Mx, int My, int stride, const double2 *__restrict__ r,
                                                          const double4 *__restrict__ dinv, float *__restrict__ img,
                                                          int height, int width, double *__restrict__ part,
                                                          const int *done) {
  if (done && *done) return;
  double acc = 0.0;
  const long long n = (long long)height * width;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int I = (int)(q / width), J = (int)(q % width);
    double su = 0.0, sv = 0.0;
    int cnt = 0;
    for (int a = 0; a < stride; ++a)
      for (int b = 0; b < stride; ++b) {
        const int i = I * stride + a, j = J * stride + b;
        if (i < Mx && j < My) {
          const size_t k = (size_t)i * My + j;
          const double4 d = dinv[k];
          const double2 rk = r[k];
          su += d.x * rk.x + d.y * rk.y;
          sv += d.z * rk.x + d.w * rk.y;
          ++cnt;
        }
      }
    if (cnt > 0) {
      su /= cnt;
      sv /= cnt;
    }
    img[q * 8 + 6] = (float)su;
    img[q * 8 + 7] = (float)sv;
    acc += su * su + sv * sv;
  }
  __shared__ double sh[PC_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < PC_THREADS / 32; ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

// rho = RMS of the residual channels (every block sums the partials in the same order);
// channels 6, 7 scaled by 1 / rho; block 0 stores rho
__global__ void __launch_bounds__(PC_THREADS) k_pc_scale(float *__restrict__ img, int height, int width,
                                                          const double *__restrict__ part, int nparts,
                                                          double *__restrict__ rho_out, const int *done) {
  if (done && *done) return;
  __shared__ double rho_sh;
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int b = 0; b < nparts; ++b) t += part[b];
    rho_sh = sqrt(t / (2.0 * (double)height * width));
    if (blockIdx.x == 0) *rho_out = rho_sh;
  }
  __syncthreads();
  const double rho = rho_sh;
  const float inv = rho > 0.0 ? (float)(1.0 / rho) : 0.0f;
  const long long n = (long long)height * width;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    img[q * 8 + 6] *= inv;
    img[q * 8 + 7] *= inv;
  }
}

// d = rho * (the network's output interpolated to the grid, as k_velocity interpolates)
__global__ void k_pc_expand(const float *__restrict__ y, int height, int width, int stride, int Mx, int My,
                            const double *__restrict__ rho, double2 *__restrict__ d, const int *done) {
  if (done && *done) return;
  const double s = *rho;
  const long long n = (long long)Mx * My;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / My), j = (int)(k % My);
    const int I0 = i / stride, J0 = j / stride;
    const int I1 = min(I0 + (i % stride ? 1 : 0), height - 1), J1 = min(J0 + (j % stride ? 1 : 0), width - 1);
    double u = 0.0, v = 0.0;
    const int Is[2] = {I0, I1}, Js[2] = {J0, J1};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const float2 o = reinterpret_cast<const float2 *>(y)[(size_t)Is[a] * width + Js[b]];
        u += (double)o.x;
        v += (double)o.y;
      }
    d[k] = make_double2(0.25 * s * u, 0.25 * s * v);
  }
}

}  // namespace pism_unet

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace pism_unet;

struct pism_gpu_unet {
  int device = 0;
  int maxB = 0, maxH = 0, maxW = 0;
  cudaStream_t stream = nullptr;
  long long nparam = 0;
  std::vector<long long> w_off, b_off, flip_off;   // offsets into the parameter / flipped arrays
  long long head_off = 0;
  float *p32 = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  bf16 *p16 = nullptr, *flip = nullptr;
  long long flip_n = 0;
  float *wg_part = nullptr;   // weight-gradient partial sums
  size_t wg_part_n = 0;
  float *small_part = nullptr;   // bias / head / loss partial sums
  float *sums = nullptr;
  float *sums_host = nullptr;
  // activations (bf16) and their gradients
  bf16 *in16 = nullptr;
  bf16 *act[NLAYERS] = {};
  bf16 *p1 = nullptr, *p2 = nullptr, *p3 = nullptr, *c3 = nullptr, *c2 = nullptr, *c1 = nullptr;
  float *y = nullptr;
  bf16 *dd1 = nullptr, *dc1 = nullptr, *dd2 = nullptr, *de1 = nullptr, *dc2 = nullptr, *dd3 = nullptr,
       *de2 = nullptr, *dc3 = nullptr, *dbt = nullptr, *de3 = nullptr, *dp3 = nullptr, *de3a = nullptr,
       *dp2 = nullptr, *de2a = nullptr, *dp1 = nullptr, *de1a = nullptr;
  int B = 0, H = 0, W = 0;   // shape of the last forward
  bool have_forward = false, have_grad = false;
  long long adam_t = 0;
  std::string err;
};

namespace {

int ufail(pism_gpu_unet *h, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  return code;
}

#define UCK(h, call)                                                                                  \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return ufail(h, PISM_GPU_SSA_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

struct UDevice {
  int prev = -1;
  explicit UDevice(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~UDevice() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int grid_for(long long n, int threads = 256) {
  return (int)std::max(1LL, std::min((n + threads - 1) / threads, 148LL * 16));
}

template <class T>
cudaError_t ualloc(T **p, size_t count) {
  return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

// level-l pixel count of a B x H x W image
inline long long pixels(int B, int H, int W, int l) { return (long long)B * (H >> l) * (W >> l); }

void conv_fwd(pism_gpu_unet *h, const bf16 *x, const bf16 *xmask, int Cin, const bf16 *w, const float *bias, int relu,
              bf16 *y, int Cout, int B, int H, int W) {
  const int tiles = B * ((H + TH - 1) / TH) * ((W + TW - 1) / TW);
  dim3 grid(tiles, Cout / NT);
  if (Cin % 32 == 0)
    k_conv3x3<32><<<grid, THREADS, 0, h->stream>>>(x, xmask, Cin, w, bias, relu, y, Cout, H, W);
  else
    k_conv3x3<16><<<grid, THREADS, 0, h->stream>>>(x, xmask, Cin, w, bias, relu, y, Cout, H, W);
}

void conv_wgrad(pism_gpu_unet *h, const bf16 *x, int Cin, const bf16 *dy, const bf16 *ymask, int Cout, int B, int H,
                int W, float *dW) {
  const int tiles = B * ((H + TH - 1) / TH) * ((W + TW - 1) / TW);
  const int ctas = std::min(tiles, WG_MAX_CTAS);
  const int CS = (Cin % 32 == 0) ? 32 : 16;
  dim3 grid(ctas, (Cout / NT) * (Cin / CS));
  if (CS == 32)
    k_conv3x3_wgrad<32><<<grid, WG_THREADS, 0, h->stream>>>(x, Cin, dy, ymask, Cout, B, H, W, h->wg_part);
  else
    k_conv3x3_wgrad<16><<<grid, WG_THREADS, 0, h->stream>>>(x, Cin, dy, ymask, Cout, B, H, W, h->wg_part);
  const int n = 9 * Cout * Cin;
  k_reduce_parts<<<grid_for(n), 256, 0, h->stream>>>(h->wg_part, ctas, n, dW);
}

void bias_grad(pism_gpu_unet *h, const bf16 *dy, const bf16 *ymask, int C, long long P, float *db) {
  const int ctas = (int)std::min<long long>(256, std::max(1LL, P / 64));
  k_bias_grad<<<ctas, 256, 0, h->stream>>>(dy, ymask, C, P, h->small_part);
  k_reduce_parts<<<1, 128, 0, h->stream>>>(h->small_part, ctas, C, db);
}

// layer l backward: X input, Y output (post-ReLU), dY given; writes dW, db and (if dX) dX
void layer_back(pism_gpu_unet *h, int l, const bf16 *X, const bf16 *Y, const bf16 *dY, bf16 *dX, int B, int H, int W) {
  const LayerDef &L = LAYERS[l];
  conv_wgrad(h, X, L.cin, dY, Y, L.cout, B, H, W, h->grad + h->w_off[l]);
  bias_grad(h, dY, Y, L.cout, (long long)B * H * W, h->grad + h->b_off[l]);
  if (dX) conv_fwd(h, dY, Y, L.cout, h->flip + h->flip_off[l], nullptr, 0, dX, L.cin, B, H, W);
}

int check_shape(pism_gpu_unet *h, int B, int H, int W) {
  if (B < 1 || H < 8 || W < 8 || H % 8 || W % 8)
    return ufail(h, PISM_GPU_SSA_EINVAL, "image %d x %d x %d: batch >= 1, height and width multiples of 8", B, H, W);
  if ((long long)B * H * W > (long long)h->maxB * h->maxH * h->maxW)
    return ufail(h, PISM_GPU_SSA_ETOOLARGE, "image %d x %d x %d exceeds the allocation (%d x %d x %d)", B, H, W,
                 h->maxB, h->maxH, h->maxW);
  return PISM_GPU_SSA_OK;
}

}  // namespace

namespace pism_unet {

void launch_features(cudaStream_t s, int Mx, int My, int stride, const double *H, const double *bed,
                     const double *tauc, const double2 *hardness, const int8_t *mask, const double2 *taud, float *out,
                     int height, int width) {
  k_features<<<grid_for((long long)height * width), 256, 0, s>>>(Mx, My, stride, H, bed, tauc, hardness, mask, taud,
                                                                  out, height, width);
}

int pc_parts(int height, int width) { return std::min(grid_for((long long)height * width, PC_THREADS), 592); }

void launch_pc_input(cudaStream_t s, int Mx, int My, int stride, const double2 *r, const double4 *dinv, float *img,
                     int height, int width, double *part, double *rho, const int *done) {
  const int nb = pc_parts(height, width);
  k_pc_image<<<nb, PC_THREADS, 0, s>>>(Mx, My, stride, r, dinv, img, height, width, part, done);
  k_pc_scale<<<nb, PC_THREADS, 0, s>>>(img, height, width, part, nb, rho, done);
}

void launch_pc_expand(cudaStream_t s, const float *y, int height, int width, int stride, int Mx, int My,
                      const double *rho, double2 *d, const int *done) {
  k_pc_expand<<<grid_for((long long)Mx * My), 256, 0, s>>>(y, height, width, stride, Mx, My, rho, d, done);
}

void launch_velocity(cudaStream_t s, const float *y, int height, int width, int stride, int Mx, int My,
                     double secpera, double2 *vel) {
  k_velocity<<<grid_for((long long)Mx * My), 256, 0, s>>>(y, height, width, stride, Mx, My, secpera, vel);
}

cudaStream_t stream_of(const pism_gpu_unet *h) { return h->stream; }
int device_of(const pism_gpu_unet *h) { return h->device; }

}  // namespace pism_unet

extern "C" {

long long pism_gpu_unet_param_count(void) { return param_count(); }

int pism_gpu_unet_create(int device, int max_batch, int max_h, int max_w, pism_gpu_unet **out) {
  if (!out || max_batch < 1 || max_h < 8 || max_w < 8 || max_h % 8 || max_w % 8) return PISM_GPU_SSA_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return PISM_GPU_SSA_ECUDA;
  UDevice dg(device);
  pism_gpu_unet *h = new pism_gpu_unet();
  h->device = device;
  h->maxB = max_batch;
  h->maxH = max_h;
  h->maxW = max_w;
  h->nparam = param_count();
  long long off = 0, foff = 0;
  for (const LayerDef &L : LAYERS) {
    h->w_off.push_back(off);
    h->flip_off.push_back(foff);
    off += 9LL * L.cout * L.cin;
    foff += 9LL * L.cout * L.cin;
    h->b_off.push_back(off);
    off += L.cout;
  }
  h->head_off = off;
  h->flip_n = foff;
  size_t wg = 0;
  for (const LayerDef &L : LAYERS) wg = std::max(wg, (size_t)9 * L.cout * L.cin);
  h->wg_part_n = wg * WG_MAX_CTAS;
  const long long P0 = (long long)max_batch * max_h * max_w;
  auto P = [&](int l) { return (size_t)(P0 >> (2 * l)); };
  int rc = PISM_GPU_SSA_OK;
  auto A = [&](bf16 **p, size_t n) {
    if (rc == PISM_GPU_SSA_OK && ualloc(p, n) != cudaSuccess) rc = PISM_GPU_SSA_ENOMEM;
  };
  auto AF = [&](float **p, size_t n) {
    if (rc == PISM_GPU_SSA_OK && ualloc(p, n) != cudaSuccess) rc = PISM_GPU_SSA_ENOMEM;
  };
  AF(&h->p32, h->nparam);
  AF(&h->grad, h->nparam);
  AF(&h->m, h->nparam);
  AF(&h->v, h->nparam);
  A(&h->p16, h->nparam);
  A(&h->flip, h->flip_n);
  AF(&h->wg_part, h->wg_part_n);
  AF(&h->small_part, 256 * 130);
  AF(&h->sums, 4);
  if (rc == PISM_GPU_SSA_OK && cudaMallocHost((void **)&h->sums_host, 4 * sizeof(float)) != cudaSuccess)
    rc = PISM_GPU_SSA_ENOMEM;
  A(&h->in16, P(0) * 16);
  for (int l = 0; l < NLAYERS; ++l) A(&h->act[l], P(LAYERS[l].level) * LAYERS[l].cout);
  A(&h->p1, P(1) * 32);
  A(&h->p2, P(2) * 64);
  A(&h->p3, P(3) * 96);
  A(&h->c3, P(2) * 224);
  A(&h->c2, P(1) * 160);
  A(&h->c1, P(0) * 96);
  AF(&h->y, P(0) * 2);
  A(&h->dd1, P(0) * 32);
  A(&h->dc1, P(0) * 96);
  A(&h->dd2, P(1) * 64);
  A(&h->de1, P(0) * 32);
  A(&h->dc2, P(1) * 160);
  A(&h->dd3, P(2) * 96);
  A(&h->de2, P(1) * 64);
  A(&h->dc3, P(2) * 224);
  A(&h->dbt, P(3) * 128);
  A(&h->de3, P(2) * 96);
  A(&h->dp3, P(3) * 96);
  A(&h->de3a, P(2) * 96);
  A(&h->dp2, P(2) * 64);
  A(&h->de2a, P(1) * 64);
  A(&h->dp1, P(1) * 32);
  A(&h->de1a, P(0) * 32);
  if (rc != PISM_GPU_SSA_OK) {
    pism_gpu_unet_destroy(h);
    return rc;
  }
  cudaMemset(h->p32, 0, h->nparam * sizeof(float));
  cudaMemset(h->p16, 0, h->nparam * sizeof(bf16));
  cudaMemset(h->flip, 0, h->flip_n * sizeof(bf16));
  cudaMemset(h->m, 0, h->nparam * sizeof(float));
  cudaMemset(h->v, 0, h->nparam * sizeof(float));
  if (cudaDeviceSynchronize() != cudaSuccess) {
    pism_gpu_unet_destroy(h);
    return PISM_GPU_SSA_ECUDA;
  }
  *out = h;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_unet_destroy(pism_gpu_unet *h) {
  if (!h) return PISM_GPU_SSA_OK;
  UDevice dg(h->device);
  cudaStreamSynchronize(h->stream);
  for (float *p : {h->p32, h->grad, h->m, h->v, h->wg_part, h->small_part, h->sums, h->y}) cudaFree(p);
  for (bf16 *p : {h->p16, h->flip, h->in16, h->p1, h->p2, h->p3, h->c3, h->c2, h->c1, h->dd1, h->dc1, h->dd2, h->de1,
                  h->dc2, h->dd3, h->de2, h->dc3, h->dbt, h->de3, h->dp3, h->de3a, h->dp2, h->de2a, h->dp1, h->de1a})
    cudaFree(p);
  for (bf16 *p : h->act) cudaFree(p);
  if (h->sums_host) cudaFreeHost(h->sums_host);
  delete h;
  return PISM_GPU_SSA_OK;
}

const char *pism_gpu_unet_last_error(const pism_gpu_unet *h) { return h ? h->err.c_str() : "null handle"; }

int pism_gpu_unet_set_stream(pism_gpu_unet *h, void *stream) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  h->stream = (cudaStream_t)stream;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_unet_set_params(pism_gpu_unet *h, const float *params, int where) {
  if (!h || !params) return PISM_GPU_SSA_EINVAL;
  UDevice dg(h->device);
  UCK(h, cudaMemcpyAsync(h->p32, params, h->nparam * sizeof(float),
                         where == PISM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
  k_to_bf16<<<grid_for(h->nparam), 256, 0, h->stream>>>(h->p32, h->nparam, h->p16);
  UCK(h, cudaMemsetAsync(h->m, 0, h->nparam * sizeof(float), h->stream));
  UCK(h, cudaMemsetAsync(h->v, 0, h->nparam * sizeof(float), h->stream));
  h->adam_t = 0;
  UCK(h, cudaGetLastError());
  UCK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_unet_get_params(pism_gpu_unet *h, float *params, int where) {
  if (!h || !params) return PISM_GPU_SSA_EINVAL;
  UDevice dg(h->device);
  UCK(h, cudaMemcpyAsync(params, h->p32, h->nparam * sizeof(float),
                         where == PISM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
  UCK(h, cudaStreamSynchronize(h->stream));
  return PISM_GPU_SSA_OK;
}

int pism_gpu_unet_forward(pism_gpu_unet *h, const float *input, int B, int H, int W, float *output) {
  if (!h || !input || !output) return PISM_GPU_SSA_EINVAL;
  int rc = check_shape(h, B, H, W);
  if (rc != PISM_GPU_SSA_OK) return rc;
  UDevice dg(h->device);
  const long long P0 = (long long)B * H * W;
  const bf16 *w = h->p16;
  const float *p = h->p32;
  auto L = [&](int l, const bf16 *x, int Hl, int Wl) {
    conv_fwd(h, x, nullptr, LAYERS[l].cin, w + h->w_off[l], p + h->b_off[l], 1, h->act[l], LAYERS[l].cout, B, Hl, Wl);
  };
  k_pack_input<<<grid_for(P0), 256, 0, h->stream>>>(input, P0, h->in16);
  L(0, h->in16, H, W);
  L(1, h->act[0], H, W);
  k_pool<<<grid_for(pixels(B, H, W, 1) * 4), 256, 0, h->stream>>>(h->act[1], 32, B, H, W, h->p1);
  L(2, h->p1, H / 2, W / 2);
  L(3, h->act[2], H / 2, W / 2);
  k_pool<<<grid_for(pixels(B, H, W, 2) * 8), 256, 0, h->stream>>>(h->act[3], 64, B, H / 2, W / 2, h->p2);
  L(4, h->p2, H / 4, W / 4);
  L(5, h->act[4], H / 4, W / 4);
  k_pool<<<grid_for(pixels(B, H, W, 3) * 12), 256, 0, h->stream>>>(h->act[5], 96, B, H / 4, W / 4, h->p3);
  L(6, h->p3, H / 8, W / 8);
  k_upcat<<<grid_for(pixels(B, H, W, 2) * 28), 256, 0, h->stream>>>(h->act[6], 128, h->act[5], 96, B, H / 4, W / 4, h->c3);
  L(7, h->c3, H / 4, W / 4);
  k_upcat<<<grid_for(pixels(B, H, W, 1) * 20), 256, 0, h->stream>>>(h->act[7], 96, h->act[3], 64, B, H / 2, W / 2, h->c2);
  L(8, h->c2, H / 2, W / 2);
  k_upcat<<<grid_for(P0 * 12), 256, 0, h->stream>>>(h->act[8], 64, h->act[1], 32, B, H, W, h->c1);
  L(9, h->c1, H, W);
  k_head<<<grid_for(P0), 256, 0, h->stream>>>(h->act[9], p + h->head_off, P0, h->y);
  UCK(h, cudaGetLastError());
  if (output != h->y)
    UCK(h, cudaMemcpyAsync(output, h->y, P0 * 2 * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
  h->B = B;
  h->H = H;
  h->W = W;
  h->have_forward = true;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_unet_backward(pism_gpu_unet *h, const float *target, const float *weight, float *loss_host,
                           float *grad_out) {
  if (!h || !target) return PISM_GPU_SSA_EINVAL;
  if (!h->have_forward) return ufail(h, PISM_GPU_SSA_ESTATE, "backward needs a forward first");
  UDevice dg(h->device);
  const int B = h->B, H = h->H, W = h->W;
  const long long P0 = (long long)B * H * W;
  // weights of the backward-data convolutions
  for (int l = 1; l < NLAYERS; ++l) {
    const int n = 9 * LAYERS[l].cout * LAYERS[l].cin;
    k_flip_weights<<<grid_for(n), 256, 0, h->stream>>>(h->p16 + h->w_off[l], LAYERS[l].cout, LAYERS[l].cin,
                                                       h->flip + h->flip_off[l]);
  }
  // loss and the head
  const int lctas = (int)std::min<long long>(256, std::max(1LL, P0 / 256));
  k_loss_parts<<<lctas, 256, 0, h->stream>>>(h->y, target, weight, P0, h->small_part);
  k_loss_finish<<<1, 32, 0, h->stream>>>(h->small_part, lctas, h->sums);
  const int hctas = (int)std::min<long long>(256, std::max(1LL, P0 / 256));
  constexpr int NG = HEAD_COUT * HEAD_CIN + HEAD_COUT;
  k_head_back<<<hctas, 256, 0, h->stream>>>(h->act[9], h->y, target, weight, h->sums, h->p32 + h->head_off, P0, h->dd1,
                                            h->small_part);
  k_reduce_parts<<<1, 128, 0, h->stream>>>(h->small_part, hctas, NG, h->grad + h->head_off);
  // decoder
  layer_back(h, 9, h->c1, h->act[9], h->dd1, h->dc1, B, H, W);
  k_upcat_back<<<grid_for(P0 * 12), 256, 0, h->stream>>>(h->dc1, 64, 32, B, H, W, h->dd2, h->de1);
  layer_back(h, 8, h->c2, h->act[8], h->dd2, h->dc2, B, H / 2, W / 2);
  k_upcat_back<<<grid_for(pixels(B, H, W, 1) * 20), 256, 0, h->stream>>>(h->dc2, 96, 64, B, H / 2, W / 2, h->dd3, h->de2);
  layer_back(h, 7, h->c3, h->act[7], h->dd3, h->dc3, B, H / 4, W / 4);
  k_upcat_back<<<grid_for(pixels(B, H, W, 2) * 28), 256, 0, h->stream>>>(h->dc3, 128, 96, B, H / 4, W / 4, h->dbt, h->de3);
  // bottleneck and encoder
  layer_back(h, 6, h->p3, h->act[6], h->dbt, h->dp3, B, H / 8, W / 8);
  k_pool_back_add<<<grid_for(pixels(B, H, W, 2) * 12), 256, 0, h->stream>>>(h->dp3, 96, B, H / 4, W / 4, h->de3);
  layer_back(h, 5, h->act[4], h->act[5], h->de3, h->de3a, B, H / 4, W / 4);
  layer_back(h, 4, h->p2, h->act[4], h->de3a, h->dp2, B, H / 4, W / 4);
  k_pool_back_add<<<grid_for(pixels(B, H, W, 1) * 8), 256, 0, h->stream>>>(h->dp2, 64, B, H / 2, W / 2, h->de2);
  layer_back(h, 3, h->act[2], h->act[3], h->de2, h->de2a, B, H / 2, W / 2);
  layer_back(h, 2, h->p1, h->act[2], h->de2a, h->dp1, B, H / 2, W / 2);
  k_pool_back_add<<<grid_for(P0 * 4), 256, 0, h->stream>>>(h->dp1, 32, B, H, W, h->de1);
  layer_back(h, 1, h->act[0], h->act[1], h->de1, h->de1a, B, H, W);
  layer_back(h, 0, h->in16, h->act[0], h->de1a, nullptr, B, H, W);
  UCK(h, cudaGetLastError());
  if (grad_out)
    UCK(h, cudaMemcpyAsync(grad_out, h->grad, h->nparam * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
  if (loss_host) {
    UCK(h, cudaMemcpyAsync(h->sums_host, h->sums, 3 * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    UCK(h, cudaStreamSynchronize(h->stream));
    *loss_host = h->sums_host[2];
  }
  h->have_grad = true;
  return PISM_GPU_SSA_OK;
}

int pism_gpu_unet_adam(pism_gpu_unet *h, float lr, float beta1, float beta2, float eps) {
  if (!h) return PISM_GPU_SSA_EINVAL;
  if (!h->have_grad) return ufail(h, PISM_GPU_SSA_ESTATE, "adam needs a backward first");
  if (!(lr > 0.0f) || !(beta1 >= 0.0f && beta1 < 1.0f) || !(beta2 >= 0.0f && beta2 < 1.0f) || !(eps > 0.0f))
    return ufail(h, PISM_GPU_SSA_EINVAL, "adam: lr > 0, 0 <= beta < 1, eps > 0");
  UDevice dg(h->device);
  h->adam_t += 1;
  const float c1 = 1.0f - std::pow(beta1, (float)h->adam_t), c2 = 1.0f - std::pow(beta2, (float)h->adam_t);
  k_adam<<<grid_for(h->nparam), 256, 0, h->stream>>>(h->p32, h->grad, h->m, h->v, h->nparam, lr, beta1, beta2, eps, c1,
                                                      c2, h->p16);
  UCK(h, cudaGetLastError());
  return PISM_GPU_SSA_OK;
}

}  // extern "C"
