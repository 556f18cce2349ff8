// ssa_internal.h — device buffers, solver state and kernel launchers of the B200
// SSAFD solver (shared by ssa_kernels.cu and ssa_capi.cu; not part of the C-ABI).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ssa_device.cuh"

namespace pism_gpu {

// Krylov status codes written by the device (KSPConvergedReason analogues)
enum : int { KSP_OK = 0, KSP_MAXIT = -3, KSP_BREAKDOWN = -5, KSP_NAN = -7 };

// scalars of one Krylov solve, owned by the device
struct KState {
  double rho, alpha, omega, beta;
  double rnorm2, bnorm2, rnorm0, rtol;
  int iter, maxit, done, status;
};

// device fields of one grid (non-owning view)
struct Fields {
  const double *H, *srf, *bed, *tauc, *melange, *gl_mask, *enthalpy, *fracture;
  const double2 *bcv;
  const int8_t *mask;
  const uint8_t *bc;
  double2 *taud, *rhs, *hardness, *nuH, *vel;
  double *beta;
  uint32_t *flags;
  double nu_bedrock;
};

// Krylov work vectors (BiCGStab)
struct Krylov {
  double2 *r, *rhat, *p, *v, *s, *t, *phat, *shat;
  double4 *dinv;
  KState *st;
};

struct Launch {
  cudaStream_t stream;
  int max_blocks;        // resident blocks (SM count x blocks per SM)
  double *partials;      // per-block partial sums (>= max_blocks * 8)
  unsigned *ticket;      // last-block ticket, kept at 0 between kernels
  long long *count;      // kernel-launch counter (may be null)
  void tick(int n = 1) const {
    if (count) *count += n;
  }
};

void launch_convert_masks(const Launch &L, int N, const double *mask, const double *bc_mask, int8_t *mask_i,
                          uint8_t *bc_i);
void launch_prepare(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, int periodicity,
                    const Fields &f);
void launch_hardness(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const Fields &f, int Mz,
                     const double *z);
void launch_nuH(const Launch &L, const GridDev &g, const pism_gpu_ssa_config &c, const Fields &f, double reg,
                double underrelax, bool with_norm, double *norm_out);
void launch_apply(const Launch &L, const GridDev &g, const Fields &f, const double2 *x, double2 *y);
void launch_diag_setup(const Launch &L, const GridDev &g, const Fields &f, double4 *dinv, int *zero_diag_cell);
void launch_bicg_init(const Launch &L, const GridDev &g, const Fields &f, const Krylov &K, const double2 *b,
                      const double2 *x);
void launch_bicg_iteration(const Launch &L, const GridDev &g, const Fields &f, const Krylov &K, double2 *x);
void launch_bfrict(const Launch &L, int N, const pism_gpu_ssa_config &c, const Fields &f, double *out);
void launch_scale(const Launch &L, int n, double a, double *x);

}  // namespace pism_gpu
