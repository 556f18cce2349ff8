// unet_internal.h — launchers shared between the network (unet.cu) and the SSA handle
// (ssa_capi.cu): the feature image built from the solver's device fields and the velocity
// built from the network's output.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

struct pism_gpu_unet;

namespace pism_unet {

void launch_features(cudaStream_t s, int Mx, int My, int stride, const double *H, const double *bed,
                     const double *tauc, const double2 *hardness, const int8_t *mask, const double2 *taud, float *out,
                     int height, int width);
void launch_velocity(cudaStream_t s, const float *y, int height, int width, int stride, int Mx, int My,
                     double secpera, double2 *vel);
// the learned preconditioner correction: the network input of a residual r (channels 0..5
// written by launch_features, 6..7 the stride x stride block means of D^-1 r divided by their
// RMS rho), and d = rho * the interpolated network output.  `part` holds pc_parts() doubles;
// `done` (may be NULL) skips the work once a Krylov solve has finished.
int pc_parts(int height, int width);
void launch_pc_input(cudaStream_t s, int Mx, int My, int stride, const double2 *r, const double4 *dinv, float *img,
                     int height, int width, double *part, double *rho, const int *done);
void launch_pc_expand(cudaStream_t s, const float *y, int height, int width, int stride, int Mx, int My,
                      const double *rho, double2 *d, const int *done);
cudaStream_t stream_of(const pism_gpu_unet *net);
int device_of(const pism_gpu_unet *net);

}  // namespace pism_unet
