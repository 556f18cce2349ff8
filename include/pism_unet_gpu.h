/* pism_unet_gpu.h — the learned warm start of the SSA solve: a small convolutional U-Net
 * (BF16 storage, FP32 accumulation) with its own forward, backward and Adam kernels.
 *
 * No reference counterpart: PISM v0.7.3 starts SSAFD::solve from the previous velocity
 * (SSA.cc:178, SSA::set_initial_guess SSA.cc:361-363).  This network predicts that initial
 * velocity from the solve's inputs; the Picard / Krylov path then iterates from it and is
 * what decides every accepted answer (the same stopping tests as from any other guess).
 *
 * Network (input 8 channels, output 2, images H x W with H, W multiples of 8):
 *   e1 = conv(conv(x, 16->32), 32->32)          full resolution  (x padded 8 -> 16 channels)
 *   e2 = conv(conv(pool(e1), 32->64), 64->64)   1/2
 *   e3 = conv(conv(pool(e2), 64->96), 96->96)   1/4
 *   b  = conv(pool(e3), 96->128)                1/8
 *   d3 = conv([up(b), e3], 224->96)             1/4
 *   d2 = conv([up(d3), e2], 160->64)            1/2
 *   d1 = conv([up(d2), e1], 96->32)             full
 *   y  = d1 . Wh + bh                           1x1, 32 -> 2, FP32 output
 * conv = 3x3 'same' (zero padding) + bias + ReLU; pool = 2x2 average; up = 2x nearest.
 *
 * Parameter vector (FP32, this order): for each of the 10 convolutions W[9][Cout][Cin]
 * (tap = 3*ky + kx, ky along the first image axis) then b[Cout]; then Wh[2][32], bh[2].
 * Layouts: images are [batch][H][W][channels], channels fastest.
 */
#ifndef PISM_UNET_GPU_H
#define PISM_UNET_GPU_H

#include "pism_ssa_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PISM_UNET_IN_CHANNELS 8
#define PISM_UNET_OUT_CHANNELS 2

typedef struct pism_gpu_unet pism_gpu_unet;   /* opaque: parameters, optimizer state, activations */

/* number of FP32 parameters */
long long pism_gpu_unet_param_count(void);

/* allocate for images up to max_batch x max_h x max_w; parameters start at zero */
int pism_gpu_unet_create(int device, int max_batch, int max_h, int max_w, pism_gpu_unet **out);
int pism_gpu_unet_destroy(pism_gpu_unet *net);
const char *pism_gpu_unet_last_error(const pism_gpu_unet *net);
int pism_gpu_unet_set_stream(pism_gpu_unet *net, void *cuda_stream);

/* parameters in the layout above; `where` is PISM_MEM_HOST or PISM_MEM_DEVICE.  Setting
 * the parameters resets the Adam moments. */
int pism_gpu_unet_set_params(pism_gpu_unet *net, const float *params, int where);
int pism_gpu_unet_get_params(pism_gpu_unet *net, float *params, int where);

/* y = f(x): input [batch][height][width][8] FP32 (device), output [batch][height][width][2]
 * FP32 (device).  Keeps the activations for a following backward. */
int pism_gpu_unet_forward(pism_gpu_unet *net, const float *input_dev, int batch, int height, int width,
                          float *output_dev);

/* Loss L = sum_{p,o} w_p (y_po - t_po)^2 / (2 sum_p w_p) of the last forward (w = 1 when
 * weight_dev is NULL) and dL/dparams.  loss_host may be NULL; grad_dev (param_count FP32,
 * device) may be NULL, the gradient stays inside for pism_gpu_unet_adam. */
int pism_gpu_unet_backward(pism_gpu_unet *net, const float *target_dev, const float *weight_dev, float *loss_host,
                           float *grad_dev);

/* one Adam step (bias-corrected moments) with the gradient of the last backward */
int pism_gpu_unet_adam(pism_gpu_unet *net, float lr, float beta1, float beta2, float eps);

/* The network's input features from an SSA handle whose inputs are set: the cells
 * (stride*I, stride*J), 0 <= I < ceil(Mx/stride), 0 <= J < ceil(My/stride), written into a
 * [height][width][8] FP32 device image (height, width >= those counts; the rest is zero).
 * Channels: H/1e3, bed/1e3, ln(max(tau_c, 1 Pa)/5e4), hardness/1e8 (0 where ice-free),
 * grounded, floating, tau_d x/1e5, tau_d y/1e5 (SI units in, driving stress computed here). */
int pism_gpu_ssa_learned_features(pism_gpu_ssa *ssa, int stride, float *features_dev, int height, int width);

/* The learned initial guess: features at `stride`, the network, velocity = 10 m/yr * sinh(y)
 * (in m/s) interpolated bilinearly back to the full grid; replaces the handle's initial guess
 * (as pism_gpu_ssa_set_initial_guess does). */
int pism_gpu_ssa_learned_guess(pism_gpu_ssa *ssa, pism_gpu_unet *net, int stride);

/* The learned preconditioner correction inside flexible GMRES (ksp_type PISM_KSP_GMRES; no
 * reference counterpart: PETSc's PCSetUp / PCApply inside KSPSolve, SSAFD.cc:136-161, 1018,
 * apply a fixed preconditioner).  With a network attached, every Arnoldi step of the handle's
 * GMRES solves takes z = M^-1 v from the configured preconditioner and then
 *   r = v - A z,   s = D^-1 r (D the 2 x 2 diagonal blocks),
 *   d = rho * N(features, s / rho)   (rho = RMS of s at the network's resolution),
 *   z += gamma d,   gamma = (r, A d) / (A d, A d),
 * the network N seeing the learned-guess features with channels 6, 7 (driving stress)
 * replaced by the stride x stride block means of s / rho, its output interpolated back to
 * the grid; gamma makes the corrected step leave no larger a residual than the
 * preconditioner alone.  Right preconditioning lets the preconditioner vary from step to step; the
 * Krylov solve's FP64 residual test decides every accepted answer as without the network.
 * net = NULL detaches it.  The network must outlive its use by the handle. */
int pism_gpu_ssa_set_learned_pc(pism_gpu_ssa *ssa, pism_gpu_unet *net, int stride);

/* The correction's network input for a residual r (device, 2N) at the current nu*H and
 * beta: a [height][width][8] FP32 device image as above (height, width >= the grid at
 * `stride`), and rho (device, one double).  For building training data. */
int pism_gpu_ssa_learned_pc_input(pism_gpu_ssa *ssa, int stride, const double *r_dev, float *image_dev, int height,
                                  int width, double *rho_dev);

#ifdef __cplusplus
}
#endif

#endif /* PISM_UNET_GPU_H */
