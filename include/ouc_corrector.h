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
 *   5 -> 32 -> 32 -> 32 -> 8 channels.
 *   inputs  (per coarse cell): Px, Pz, Sx, Sz of the current level divided
 *           by the state's scale s, and Vp/Vs - 1.7;
 *   outputs: corrections of Px, Pz, Sx, Sz at the current and the previous
 *           level, in units of s.
 * Convolutions run as implicit GEMMs on the tensor cores (tcgen05, BF16
 * operands, FP32 accumulation in tensor memory); the input-gradient pass is
 * the same kernel on the flipped, transposed weights; weight gradients
 * accumulate in FP32.
 *
 * Parameters (FP32 master copy, ouc_cnn_nparams() floats): for each layer l
 * in order, W_l[cout][cin][5][5] (kx, kz: x-major as the grids) then b_l[cout].
 * Images are NHWC: [n][H][W][C] float32, H along x, W along z.
 */
#ifndef OUC_CORRECTOR_H
#define OUC_CORRECTOR_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ouc_cnn ouc_cnn;

#define OUC_CNN_IN 5
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
/* Non-zero when a bounded wait inside a corrector kernel ran out (the
 * affected outputs are then invalid); cleared by this call. */
int ouc_cnn_error(ouc_cnn* net);

#ifdef __cplusplus
}
#endif
#endif /* OUC_CORRECTOR_H */
