// ssa_noalloc.cu — pism_gpu_ssa_nuH_noalloc: nu*H, the basal drag coefficient and the
// two L1 norms of the Picard convergence test, computed without allocating any memory.
//
// Why: some callers cannot call cudaMalloc at all — a host that hands every
// allocation to its own pool or arena, code running under a memory budget that
// forbids new device allocations, or a language binding with no access to the
// CUDA allocator.  The handle API allocates its scratch in
// pism_gpu_ssa_create; this entry point instead keeps its scratch in the fixed
// file-scope device array below, so the caller passes only inputs and outputs.
//
// The scratch holds the partial sums of at most NOALLOC_MAX_BLOCKS blocks and the last-block
// ticket.  The kernel's blocks walk the grid's 32 x 8-cell tiles with a stride of the block
// count, so every grid shape of up to PISM_GPU_SSA_NOALLOC_MAX_CELLS cells fits, however
// thin; larger grids are rejected.  Every GPU that loads this library holds the array
// (512 KiB) until the process exits.
#include <mutex>

#include "ssa_device.cuh"

namespace pism_gpu {
namespace {

constexpr int TJn = 32, TIn = 8, NTn = TJn * TIn;
constexpr int NOALLOC_MAX_BLOCKS = PISM_GPU_SSA_NOALLOC_MAX_CELLS / NTn;
constexpr int NV = 4;   // |nuH_0|, |nuH_1|, |change_0|, |change_1|

// partial sums of every block, then the ticket in the last slot
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_BLOCKS * NV + 1];

__device__ __forceinline__ double warp_sum_n(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int as_int(double m) { return (int)floor(m + 0.5); }   // IceModelVec_inline.hh:94-100

struct Params {
  double reg, underrelax, Hmin, notional, schoof_reg, visc_power, enh_scaling, area;
};

// compute_nuH_staggered (SSAFD.cc:1359-1421) + under-relaxation (SSAFD.cc:1061-1064) +
// compute_nuH_norm (SSAFD.cc:1170-1189) + the drag of SSAFD.cc:744-759; each block takes the
// tiles blockIdx.x, blockIdx.x + gridDim.x, ...
__global__ void __launch_bounds__(NTn) k_nuH_noalloc(GridDev g, int tiles_j, int tiles, pism_gpu_ssa_config c,
                                                     Params p, const double2 *__restrict__ vel,
                                                     const double *__restrict__ H,
                                                     const double2 *__restrict__ hardness,
                                                     const double *__restrict__ mask, const double *__restrict__ tauc,
                                                     const double *__restrict__ gl_mask, double2 *__restrict__ nuH,
                                                     double *__restrict__ beta, double *scratch, double *norms) {
  double acc[NV] = {0.0, 0.0, 0.0, 0.0};
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int ti = tile / tiles_j, tj = tile - ti * tiles_j;
    const int j = tj * TJn + (threadIdx.x & (TJn - 1)), i = ti * TIn + (threadIdx.x >> 5);
    if (i < g.Mx && j < g.My) {
      const double dx = g.dx, dy = g.dy;
      const int k = cell(g, i, j);
      const double2 uc = vel[k], ue = vel[nbr(g, i, j, 1, 0)], un = vel[nbr(g, i, j, 0, 1)],
                    us = vel[nbr(g, i, j, 0, -1)], uw = vel[nbr(g, i, j, -1, 0)], une = vel[nbr(g, i, j, 1, 1)],
                    use = vel[nbr(g, i, j, 1, -1)], unw = vel[nbr(g, i, j, -1, 1)];
      const double Hc = H[k];
      const double2 B = hardness[k];
      double r[2];
      for (int o = 0; o < 2; ++o) {
        const double Hf = 0.5 * (Hc + H[nbr(g, i, j, 1 - o, o)]);
        if (Hf < p.Hmin) {
          r[o] = p.notional;
          continue;
        }
        double u_x, u_y, v_x, v_y;
        if (o == 0) {
          u_x = (ue.x - uc.x) / dx;
          u_y = (un.x + une.x - us.x - use.x) / (4 * dy);
          v_x = (ue.y - uc.y) / dx;
          v_y = (un.y + une.y - us.y - use.y) / (4 * dy);
        } else {
          u_x = (ue.x + une.x - uw.x - unw.x) / (4 * dx);
          u_y = (un.x - uc.x) / dy;
          v_x = (ue.y + une.y - uw.y - unw.y) / (4 * dx);
          v_y = (un.y - uc.y) / dy;
        }
        const double Bo = o == 0 ? B.x : B.y;
        const double nu = 0.5 * Bo * pow(p.schoof_reg + second_invariant_2d(u_x, u_y, v_x, v_y), p.visc_power);
        r[o] = nu * Hf;
        r[o] *= p.enh_scaling;
        r[o] += p.reg;
      }
      const double2 old = nuH[k];
      if (p.underrelax != 1.0) {
        r[0] *= p.underrelax;
        r[0] += (1.0 - p.underrelax) * old.x;
        r[1] *= p.underrelax;
        r[1] += (1.0 - p.underrelax) * old.y;
      }
      nuH[k] = make_double2(r[0], r[1]);
      // L1 over the ghosted local vector: periodic ghost copies of the edge cells count again
      const double w = ((i == 0 ? 1.0 : 0.0) + (i == g.Mx - 1 ? 1.0 : 0.0) + 1.0) *
                       ((j == 0 ? 1.0 : 0.0) + (j == g.My - 1 ? 1.0 : 0.0) + 1.0);
      acc[0] += fabs(r[0]) * w;
      acc[1] += fabs(r[1]) * w;
      acc[2] += fabs(old.x - r[0]) * w;
      acc[3] += fabs(old.y - r[1]) * w;
      const int M = as_int(mask[k]);
      double bta = 0.0;
      if (m_grounded_ice(M))
        bta = basal_drag(c, tauc[k], uc.x, uc.y);
      else if (m_ice_free_land(M))
        bta = c.beta_ice_free_bedrock;
      if (c.sub_groundingline && m_icy(M)) bta = gl_mask[k] * basal_drag(c, tauc[k], uc.x, uc.y);
      beta[k] = bta;
    }
  }
  // block sums -> scratch; the last block adds them in block order
  __shared__ double sh[NV][NTn / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int v = 0; v < NV; ++v) {
    const double s = warp_sum_n(acc[v]);
    if (lane == 0) sh[v][warp] = s;
  }
  __syncthreads();
  unsigned *ticket = reinterpret_cast<unsigned *>(&scratch[NOALLOC_MAX_BLOCKS * NV]);
  if (threadIdx.x == 0) {
    for (int v = 0; v < NV; ++v) {
      double s = 0.0;
      for (int q = 0; q < NTn / 32; ++q) s += sh[v][q];
      scratch[blockIdx.x * NV + v] = s;
    }
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int v = 0; v < NV; ++v) {
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += NTn) s += __ldcg(&scratch[b * NV + v]);
    s = warp_sum_n(s);
    if (lane == 0) sh[v][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[NV];
    for (int v = 0; v < NV; ++v) {
      t[v] = 0.0;
      for (int q = 0; q < NTn / 32; ++q) t[v] += sh[v][q];
      t[v] *= p.area;
    }
    norms[0] = sqrt(t[0] * t[0] + t[1] * t[1]);
    norms[1] = sqrt(t[2] * t[2] + t[3] * t[3]);
    *ticket = 0u;
  }
}

std::mutex g_setup_mutex;
constexpr int MAX_DEVICES = 64;
double *g_scratch_addr[MAX_DEVICES] = {nullptr};

}  // namespace
}  // namespace pism_gpu

using namespace pism_gpu;

extern "C" int pism_gpu_ssa_nuH_noalloc(const pism_gpu_grid *grid, const pism_gpu_ssa_config *cfg,
                                        const double *velocity, const double *thickness,
                                        const double *hardness_stag, const double *mask, const double *tauc,
                                        const double *gl_mask, double nuH_regularization, double underrelax,
                                        double *nuH, double *beta, double *norms, void *cuda_stream) {
  if (!grid || !cfg || !velocity || !thickness || !hardness_stag || !mask || !tauc || !nuH || !beta || !norms)
    return PISM_GPU_SSA_EINVAL;
  if (grid->Mx < 3 || grid->My < 3 || !(grid->dx > 0) || !(grid->dy > 0)) return PISM_GPU_SSA_EINVAL;
  if (cfg->calving_front_stress_boundary_condition) return PISM_GPU_SSA_EINVAL;   // plain stencil only
  if (cfg->sub_groundingline && !gl_mask) return PISM_GPU_SSA_EINVAL;
  if ((long long)grid->Mx * grid->My > PISM_GPU_SSA_NOALLOC_MAX_CELLS) return PISM_GPU_SSA_ETOOLARGE;
  const int tiles_j = (grid->My + TJn - 1) / TJn;
  const int tiles = tiles_j * ((grid->Mx + TIn - 1) / TIn);   // < 2^31: Mx, My >= 3, cells <= 2^22
  const int blocks = tiles < NOALLOC_MAX_BLOCKS ? tiles : NOALLOC_MAX_BLOCKS;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return PISM_GPU_SSA_ECUDA;
  double *scratch;
  {
    // set-up, once per device, with that device current: the array's name is a
    // host-side stand-in, so the kernel is given the device address instead
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PISM_GPU_SSA_ECUDA;
      g_scratch_addr[dev] = static_cast<double *>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t stream = (cudaStream_t)cuda_stream;
  // the ticket must start at zero; a previous call leaves it at zero, an aborted one may not
  if (cudaMemsetAsync(&scratch[NOALLOC_MAX_BLOCKS * NV], 0, sizeof(double), stream) != cudaSuccess)
    return PISM_GPU_SSA_ECUDA;
  GridDev g{grid->Mx, grid->My, grid->dx, grid->dy};
  const double n = cfg->ssa_Glen_exponent, sv = cfg->Schoof_regularizing_velocity / cfg->Schoof_regularizing_length;
  Params p{nuH_regularization,
           underrelax,
           cfg->min_thickness_strength_extension_ssa,
           cfg->constant_nu_strength_extension_ssa * cfg->min_thickness_strength_extension_ssa,
           sv * sv,
           (1.0 - n) / (2.0 * n),
           1.0 / pow(cfg->ssa_enhancement_factor, 1.0 / n),
           grid->dx * grid->dy};
  // launched through cudaLaunchKernel, whose return value is this launch's own status: an
  // error that earlier work of the caller left pending is neither read nor cleared here
  const double2 *vel2 = (const double2 *)velocity, *hard2 = (const double2 *)hardness_stag;
  double2 *nuH2 = (double2 *)nuH;
  void *args[] = {&g, (void *)&tiles_j, (void *)&tiles, (void *)cfg, &p, &vel2, (void *)&thickness, &hard2,
                  (void *)&mask, (void *)&tauc, (void *)&gl_mask, &nuH2, &beta, &scratch, &norms};
  const cudaError_t e = cudaLaunchKernel((const void *)k_nuH_noalloc, dim3((unsigned)blocks), dim3(NTn), args, 0,
                                         stream);
  return e == cudaSuccess ? PISM_GPU_SSA_OK : PISM_GPU_SSA_ECUDA;
}
