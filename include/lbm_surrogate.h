/* lbm_surrogate.h -- device kernels of the learned warm start.
 *
 * The reference has no counterpart: it always starts from the conduction
 * state of initial() (natural-convection_2dim_mono.f90:199-240).  These
 * entry points are the forward and backward passes of a small convolutional
 * network (4-level U-Net) that predicts steady (u, v, T) fields from
 * (Ra, Pr, grid-coordinate maps); its prediction seeds lbm_init_warm().
 *
 * Conventions
 *   - images are NHWC: element (b, y, x, c) of a tensor with channel stride
 *     cs and channel offset co lives at ((b*H + y)*W + x)*cs + co + c, so one
 *     buffer can hold a channel concatenation (a U-Net skip connection);
 *   - activations and weights are bfloat16 (passed as void *), products are
 *     accumulated in FP32; gradients and optimizer state are FP32;
 *   - 3x3 weights are [Cout][9][Cin] with tap = 3*ky + kx, padding 1, stride 1;
 *   - bf16 tensors read by the 3x3 kernels need 16-byte aligned rows:
 *     channel stride, channel offset multiples of 8 and Cin a multiple of 32;
 *   - every call is asynchronous on `stream` (a cudaStream_t, NULL = legacy
 *     default) and returns LBM_OK or a negative LBM_ERR_* status
 *     (include/lbm_b200.h); lbm_last_error() has the message.
 */
#ifndef LBM_SURROGATE_H
#define LBM_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* z = conv3x3(x, w) + bias over B images of H x W.
 *   of  (FP32, stride os, offset oo): receives z, or z is added to it when
 *       accumulate != 0 (then bias must be NULL); may be NULL;
 *   oa  (bf16, stride as, offset ao): receives act(z) (act 0: identity,
 *       1: SiLU z*sigmoid(z)); may be NULL; not allowed with accumulate.
 * With x = dL/dz of a layer and w = lbm_nn_flip_weights() of its weights the
 * same call is the data gradient of that layer. */
int lbm_nn_conv3x3(const void *x, int64_t xs, int32_t xo, const void *w, const float *bias,
                   int32_t B, int32_t H, int32_t W, int32_t Cin, int32_t Cout,
                   float *of, int64_t os, int32_t oo, int32_t accumulate,
                   void *oa, int64_t as, int32_t ao, int32_t act, void *stream);

/* wt[ci][tap][co] = w[co][8 - tap][ci]: the weights of the data gradient. */
int lbm_nn_flip_weights(const void *w, void *wt, int32_t Cout, int32_t Cin, void *stream);

/* dw[co][tap][ci] = sum over pixels p of dz[p][co] * x[p + offset(tap)][ci]
 * (dz contiguous, Cout channels).  ws: FP32 scratch of ws_elems elements
 * (lbm_nn_wgrad_workspace gives the size).  Deterministic. */
int64_t lbm_nn_wgrad_workspace(int32_t B, int32_t H, int32_t W, int32_t Cin, int32_t Cout);
int lbm_nn_conv3x3_wgrad(const void *dz, const void *x, int64_t xs, int32_t xo,
                         int32_t B, int32_t H, int32_t W, int32_t Cin, int32_t Cout,
                         float *ws, int64_t ws_elems, float *dw, void *stream);

/* out[c] = sum over rows p < P of a[p][c] (bf16, contiguous C channels):
 * the bias gradient.  ws: FP32 scratch of lbm_nn_colsum_workspace(P, C). */
int64_t lbm_nn_colsum_workspace(int64_t P, int32_t C);
int lbm_nn_colsum(const void *a, int64_t P, int32_t C, float *ws, float *out, void *stream);

/* dz[p][c] (bf16, contiguous) = da[p*das + dao + c] * silu'(z[p][c]). */
int lbm_nn_silu_backward(const float *da, int64_t das, int32_t dao, const float *z,
                         int64_t P, int32_t C, void *dz, void *stream);

/* 2x2 average pooling of x (B, H, W even) into y (B, H/2, W/2); bf16. */
int lbm_nn_pool2(const void *x, int64_t xs, int32_t xo, int32_t B, int32_t H, int32_t W, int32_t C,
                 void *y, int64_t ys, int32_t yo, void *stream);
/* dx (B, H, W) += pool2 backward of dy (B, H/2, W/2); FP32. */
int lbm_nn_pool2_backward(const float *dy, int64_t dys, int32_t dyo, int32_t B, int32_t H, int32_t W,
                          int32_t C, float *dx, int64_t dxs, int32_t dxo, void *stream);

/* Nearest-neighbour 2x upsampling of x (B, h, w) into y (B, 2h, 2w); bf16. */
int lbm_nn_up2(const void *x, int64_t xs, int32_t xo, int32_t B, int32_t h, int32_t w, int32_t C,
               void *y, int64_t ys, int32_t yo, void *stream);
/* dx (B, h, w) = (accumulate ? dx : 0) + sum of the 2x2 block of dy; FP32. */
int lbm_nn_up2_backward(const float *dy, int64_t dys, int32_t dyo, int32_t B, int32_t h, int32_t w,
                        int32_t C, float *dx, int64_t dxs, int32_t dxo, int32_t accumulate, void *stream);

/* 1x1 output layer: y[p][j] = sum_c a[p][c] wh[j][c] + bh[j], j < J <= 8
 * (a, wh bf16; bh, y FP32; y contiguous). */
int lbm_nn_head(const void *a, int64_t as, int32_t ao, const void *wh, const float *bh,
                int64_t P, int32_t C, int32_t J, float *y, void *stream);
/* Its backward: da (FP32, stride das, offset dao) = dy wh;
 * dwh = dy^T a and dbh = column sums of dy (deterministic; ws of
 * lbm_nn_head_workspace(P, C, J) FP32 elements). */
int64_t lbm_nn_head_workspace(int64_t P, int32_t C, int32_t J);
int lbm_nn_head_backward(const float *dy, const void *a, int64_t as, int32_t ao, const void *wh,
                         int64_t P, int32_t C, int32_t J, float *da, int64_t das, int32_t dao,
                         float *ws, int64_t ws_elems, float *dwh, float *dbh, void *stream);

/* Weighted mean squared error over P x J values:
 *   loss = sum_{p,j} cw[j] (y - t)^2 / (P J),  dy = 2 cw[j] (y - t) / (P J)
 * (all FP32; loss is one device float; ws of lbm_nn_mse_workspace(P, J)). */
int64_t lbm_nn_mse_workspace(int64_t P, int32_t J);
int lbm_nn_mse(const float *y, const float *t, const float *cw, int64_t P, int32_t J, float *dy,
               float *ws, int64_t ws_elems, float *loss, void *stream);

/* One Adam step over n parameters (FP32 master p, bf16 copy pb refreshed):
 *   m = b1 m + (1-b1) g;  v = b2 v + (1-b2) g^2;
 *   p -= lr * ((m / c1) / (sqrt(v / c2) + eps) + wd p)
 * with c1 = 1 - b1^t, c2 = 1 - b2^t from the caller. */
int lbm_nn_adam(float *p, void *pb, const float *g, float *m, float *v, int64_t n, float lr, float b1,
                float b2, float eps, float c1, float c2, float wd, void *stream);

/* Which tensor-core path lbm_nn_conv3x3 uses: 0 mma.sync (m16n8k16, the
 * default: faster on the network's layer sizes), 1 tcgen05 with the
 * accumulator in tensor memory.  Both give the same results to bf16 rounding.
 * Process-wide. */
int lbm_nn_set_tensor_path(int32_t path);
int lbm_nn_get_tensor_path(void);

/* Number of tcgen05 convolution blocks that gave up on a bounded wait (their
 * output is then incomplete); reset != 0 clears the count.  Synchronous. */
int lbm_nn_timeouts(int32_t *count, int32_t reset);

/* Round FP32 to bf16 (n elements). */
int lbm_nn_to_bf16(const float *x, void *y, int64_t n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LBM_SURROGATE_H */
