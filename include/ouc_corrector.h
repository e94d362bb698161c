/*
 * ouc_corrector.h -- C ABI of the learned dispersion corrector (libouc.so).
 *
 * No counterpart in the reference.  A coarse run (half-order N = 2 at twice
 * the fine spacing and time step) disperses; a small CNN, applied every
 * `every` coarse steps, predicts the difference between the coarse state
 * and the fine (N = 5) solution sampled onto the coarse grid, and the
 * correction is added to the coarse wavefield.
 *
 * Network: four 5x5 convolutions, "same" zero padding, ReLU between them:
 *   10 -> 32 -> 32 -> 32 -> 8 channels (the first layer pads to 16 inputs).
 *   inputs  (per coarse cell, the whole leapfrog state): Px, Pz, Sx, Sz at
 *           the current level over s_d; their change over the last step
 *           (the particle velocity of the P and S parts times dt) over s_v;
 *           Vp/Vs - 1.7 and Vp dt/h - 0.5, both times the local motion
 *           (the sum of |velocity inputs|) -- s_d and s_v are the largest |U|
 *           and |U^n - U^(n-1)| on the interior;
 *   outputs: the correction of Px, Pz, Sx, Sz at the current leapfrog level
 *           (units s_d / 16) and of their change over the last step (units
 *           s_v / 16), applied as U^n += s_d c_U / 16 and
 *           U^(n-1) += (s_d c_U - s_v c_V) / 16 on the interior less a band
 *           of 4 cells along the absorbing layers and a disc of radius 6
 *           cells around the source, after a low-pass S (the binomial filter
 *           (1 4 6 4 1)/16 along x and along z): the corrector works in the
 *           band the coarse grid resolves.
 * The learned path trains and runs the network without biases (they stay
 * zero), so a region at rest receives no correction.
 * Convolutions run as implicit GEMMs on the tensor cores (tcgen05, BF16
 * operands, FP32 accumulation in tensor memory); the input-gradient pass is
 * the same kernel on the flipped, transposed weights; weight gradients are
 * tensor-core GEMMs over the pixels (BF16 operands, FP32 accumulation),
 * reduced across CTAs in a fixed order, so training is reproducible.
 *
 * Parameters (FP32 master copy, ouc_cnn_nparams() floats): for each layer l
 * in order, W_l[cout][cin][5][5] (kx, kz: x-major as the grids) then b_l[cout].
 * Images are NHWC: [n][H][W][C] float32, H along x, W along z.
 */
#ifndef OUC_CORRECTOR_H
#define OUC_CORRECTOR_H

#include <stddef.h>

#include "ouc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ouc_cnn ouc_cnn;

#define OUC_CNN_IN 10
#define OUC_CNN_WIDTH 32
#define OUC_CNN_OUT 8

int ouc_cnn_nparams(void);
int ouc_cnn_create(int device, ouc_cnn** out);
int ouc_cnn_destroy(ouc_cnn* net);
int ouc_cnn_set_params(ouc_cnn* net, const float* params);   /* host, ouc_cnn_nparams() floats */
int ouc_cnn_get_params(const ouc_cnn* net, float* params);

/* Forward: d_in [n][H][W][5] -> d_out [n][H][W][8], device float32.  Keeps
 * the activations of the last call for ouc_cnn_backward_dev. */
int ouc_cnn_forward_dev(ouc_cnn* net, int n, int H, int W, const float* d_in, float* d_out, void* stream);
/* Backward of the last forward: d_gout = dLoss/d_out [n][H][W][8]; adds the
 * parameter gradients into the network's gradient buffer. */
int ouc_cnn_backward_dev(ouc_cnn* net, const float* d_gout, void* stream);
int ouc_cnn_zero_grad(ouc_cnn* net, void* stream);
int ouc_cnn_get_grads(const ouc_cnn* net, float* grads);      /* host, ouc_cnn_nparams() floats */
/* One Adam step (Kingma & Ba, 2015) on the accumulated gradients. */
int ouc_cnn_adam_step(ouc_cnn* net, float lr, float beta1, float beta2, float eps, void* stream);
/* Train on npairs device pairs: d_in [npairs][H][W][OUC_CNN_IN], d_tgt
 * [npairs][H][W][8].  Each epoch visits the pairs in a seeded random order in
 * minibatches of `batch`; the loss is the mean squared error over the
 * rectangle [i0, i1) x [j0, j1) of each image (elsewhere the gradient is
 * zero), minimised by Adam (beta 0.9 / 0.999) with the bias gradients held at
 * zero.  epoch_loss (host, `epochs` floats, may be NULL) receives the mean
 * minibatch loss of each epoch.  Allocates its minibatch buffers. */
int ouc_cnn_train(ouc_cnn* net, const float* d_in, const float* d_tgt, int npairs, int H, int W, int i0, int i1,
                  int j0, int j1, int batch, int epochs, float lr, unsigned seed, float* epoch_loss, void* stream);

/* ---- the learned coarse path (ouc.h contexts) ---------------------------
 * A coarse context has half the cells of a fine one in each direction (npml
 * halved too), twice the spacing and twice the time step; coarse padded cell
 * (i, j) lies where fine padded cell (2i, 2j) does.  Fine shots sit on even
 * interior cells; the coarse shot is the fine one halved. */

/* Coarse wavelet from the fine one: out[m] = fine[2m] / 4 (the coarse
 * source cell has four times the fine cell's area). */
int ouc_coarse_wavelet(const float* fine, int nt_coarse, float* out);

/* Coarse forward modeling with the corrector applied after every `every`
 * steps (net NULL: the plain coarse run).  Gathers X*nt in the context's
 * gather layout (host, either may be NULL); the wavelet is the coarse one. */
int ouc_forward_learned(ouc_ctx* ctx, ouc_cnn* net, const ouc_shot* shot, const float* wavelet, int every,
                        float* gather_vx, float* gather_vz);

/* Fine forward modeling sampled as the coarse grid sees it: gathers of the
 * restricted displacement (cubic midpoint interpolation along the staggered
 * direction) at the coarse receiver row, every second fine step; (X/2) x
 * nt_coarse each in the fine context's gather layout.  The spot check of
 * the learned path compares against these. */
int ouc_forward_restricted(ouc_ctx* fine, const ouc_shot* shot, const float* wavelet, int nt_coarse,
                           float* gather_vx, float* gather_vz);

/* Training pairs of one shot: the fine run (wavelet: the fine one) and the
 * coarse run advance together; at every `every`-th coarse level m the coarse
 * state gives the network input and its difference d from the restricted fine
 * state the target (correction region only): S of 16 d^m / s_d and of
 * 16 (d^m - d^(m-1)) / s_v.  With net NULL every interval starts from the
 * restricted fine state (teacher forcing); otherwise from the coarse state
 * corrected by `net` (on-policy pairs: the states the corrected run visits).
 * noise > 0 perturbs each input state on the correction region by uniform
 * noise of that size relative to s_d and s_v (seeded by `seed`), so that the
 * network learns to remove perturbations it did not cause.  Pairs without
 * motion are skipped.  Writes at most max_pairs pairs into
 * d_in [.][X_c][Z_c][OUC_CNN_IN] and d_tgt [.][X_c][Z_c][8] (device) and
 * their count into *npairs. */
int ouc_learned_pairs(ouc_ctx* fine, ouc_ctx* coarse, ouc_cnn* net, const ouc_shot* shot, const float* wavelet,
                      int every, float noise, unsigned seed, int max_pairs, float* d_in, float* d_tgt, int* npairs);

/* Non-zero when a bounded wait inside a corrector kernel ran out (the
 * affected outputs are then invalid); cleared by this call. */
int ouc_cnn_error(ouc_cnn* net);

#ifdef __cplusplus
}
#endif
#endif /* OUC_CORRECTOR_H */
