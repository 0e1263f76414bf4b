/* pcom_cnn.h -- C ABI of the learned subgrid closure (no counterpart in the
 * reference, which has no learned component).
 *
 * A 5-layer 3x3 convolutional network over images of H x W pixels (one image
 * per model level of the coarse grid, NHWC, channels contiguous):
 *   in 16 (5 used: u, v, T, S, specific-volume anomaly; BF16)
 *   -> 64 -> 64 -> 64 -> 64 (ReLU, BF16 activations)
 *   -> out 4 (du, dv, dT, dS tendency residuals, FP32).
 * Zero padding in y, wrap-around in x when periodic_x.  Every convolution
 * (forward, data and weight gradients) runs on the tensor cores (tcgen05,
 * BF16 operands, FP32 accumulation).
 *
 * Parameters, FP32, in this order per layer l = 1..5: W_l [9][N_l][K_l]
 * (tap t = 3 (dy + 1) + (dx + 1), output channel, input channel; K
 * contiguous) then b_l [N_l], with (K_l, N_l) = (16, 64), (64, 64), (64, 64),
 * (64, 64), (64, 16).  Input channels 5..15 of layer 1 and output channels
 * 4..15 of layer 5 are padding and are kept at zero.
 *
 * Device pointers throughout; calls run on the network's stream (its own,
 * or the one given to pcom_cnn_set_stream) and are synchronous on return
 * unless named _async. */
#ifndef PCOM_CNN_H
#define PCOM_CNN_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCOM_CNN_OK 0
#define PCOM_CNN_ERR_ARG 1
#define PCOM_CNN_ERR_CUDA 2
#define PCOM_CNN_ERR_TIMEOUT 5

typedef struct pcom_cnn pcom_cnn;

int pcom_cnn_last_error(char *buf, int32_t len);
int64_t pcom_cnn_param_count(void);
/* Buffers for up to max_images images of H x W. */
int pcom_cnn_create(int32_t H, int32_t W, int32_t max_images, int32_t periodic_x, pcom_cnn **out);
int pcom_cnn_destroy(pcom_cnn *c);
/* Run on a caller's stream (stays the caller's: never destroyed here), or
 * with stream = NULL on a new stream of the network's own. */
int pcom_cnn_set_stream(pcom_cnn *c, void *stream);
/* Host FP32 parameters in the layout above (resets the Adam moments). */
int pcom_cnn_set_params(pcom_cnn *c, const float *params, int64_t n);
int pcom_cnn_get_params(pcom_cnn *c, float *params, int64_t n);
/* x: BF16 [nimg][H][W][16]; y: FP32 [nimg][H][W][4]. */
int pcom_cnn_forward(pcom_cnn *c, const void *x, float *y, int32_t nimg);
int pcom_cnn_forward_async(pcom_cnn *c, const void *x, float *y, int32_t nimg);
/* Loss = sum mask (y - target)^2 / sum mask over [nimg][H][W][4] (FP32
 * target and mask); its gradient with respect to every parameter (host
 * FP32, parameter layout) and the loss. */
int pcom_cnn_gradient(pcom_cnn *c, const void *x, const float *target, const float *mask, int32_t nimg,
                      float *grad_host, double *loss);
/* One Adam step (lr; beta1 0.9, beta2 0.999, eps 1e-8) on that loss. */
int pcom_cnn_train_step(pcom_cnn *c, const void *x, const float *target, const float *mask, int32_t nimg, float lr,
                        double *loss);
/* One tensor-core convolution layer, for checks against a CPU convolution:
 * out[p][n] = sum_t sum_c in[src(p, t)][c] w[t][n][c] with mode 0 (+ bias,
 * ReLU, BF16 out), 1 (+ bias, FP32 out, first nstore channels) or 2 (times
 * (aux > 0), BF16 out); (cin, nout) in {(16,64), (64,64), (64,16), (16,16)}. */
int pcom_cnn_conv_layer(int32_t cin, int32_t nout, const void *in, const void *w, const float *bias, const void *aux,
                        void *out, int64_t npix, int32_t H, int32_t W, int32_t periodic_x, int32_t mode, int32_t nstore,
                        void *stream);
/* dw[t][n][c] += sum_p in[src(p, t)][c] g[p][n] (FP32 dw); (cin, nout) in
 * {(16,64), (64,64), (64,16)}. */
int pcom_cnn_wgrad_layer(int32_t cin, int32_t nout, const void *in, const void *g, float *dw, int64_t npix, int32_t H,
                         int32_t W, int32_t periodic_x, void *stream);

#ifdef __cplusplus
}
#endif
#endif
