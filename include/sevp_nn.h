/*
 * sevp_nn.h -- C ABI of the learned warm start of libsevp_b200.so.
 *
 * None of these entry points replaces a reference routine: the reference
 * has no learned component.  They are the building blocks of the U-Net that
 * predicts the next time step's solution (musoc_solver_b200/unet.py and
 * warmstart.py assemble the network from them) and of its coupling to a
 * solver context (sevp_b200.h) through sevp_set_warmstart.
 *
 * Tensors are NHWC BF16 [B][H][W][ld] with a layer's channels at channel
 * offset `off` inside the leading dimension `ld` (a decoder's concatenated
 * input is one buffer that two producers write).  All pointers are device
 * pointers; `stream` is a cudaStream_t (NULL: legacy default stream).  Every
 * function returns a SEVP_* status (sevp_b200.h) and only enqueues work.
 */
#ifndef SEVP_NN_H
#define SEVP_NN_H

#include "sevp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* 3x3 convolution, zero padding, on warp-level tensor-core MMA:
 *   out[p][out_off + co] = act(bias[co] + sum_{tap, ci} in'[p + shift(tap)][ci] * w[tap][ci][co])
 * w is [9][cin][cout].  flip != 0 mirrors the tap of the input shift (the
 * data gradient, called with the transposed weights [9][cout][cin]); mask
 * (optional) zeroes input values whose mask entry is <= 0 (ReLU backward).
 * act = ReLU when relu != 0.  cin, cout multiples of 16. */
int sevp_nn_conv3x3(const void *in, int in_ld, int in_off, int cin, const void *w,
                    const float *bias, void *out, int out_ld, int out_off, int cout, int B, int H,
                    int W, int relu, const void *mask, int mask_ld, int mask_off, int flip,
                    void *stream);

/* Forward 3x3 convolution on the tcgen05 tensor cores (FP32 accumulator in
 * tensor memory): the same result as sevp_nn_conv3x3 with flip = 0 and no
 * mask, with the K-major weights wk = [9][cout][cin].  cin in {16, 32, 64,
 * 128, 256}; cout a multiple of 16 up to 256; ld and off multiples of 8;
 * pointers 16-byte aligned. */
int sevp_nn_conv3x3_tc(const void *in, int in_ld, int in_off, int cin, const void *wk,
                       const float *bias, void *out, int out_ld, int out_off, int cout, int B,
                       int H, int W, int relu, void *stream);

/* The same forward convolution with both operands loaded by TMA (tensor-map
 * loads with hardware zero fill at the image edges, 128-byte swizzle) and a
 * warp-specialised producer / MMA issuer; tiles are 128 pixels of one image
 * row.  cin in {16, 32, 64, 128, 192, 256}, other limits as above. */
int sevp_nn_conv3x3_tma(const void *in, int in_ld, int in_off, int cin, const void *wk,
                        const float *bias, void *out, int out_ld, int out_off, int cout, int B,
                        int H, int W, int relu, void *stream);

/* First error code (SEVP_TIMEOUT) a tensor-core kernel recorded since the
 * last call, 0 if none; clears it.  Synchronises the device. */
int sevp_nn_tc_status(int *code);
/* Test hook for the bounded waits of sevp_nn_conv3x3_tma: the number of
 * polls its load and MMA waits make before giving up (0: give up at once;
 * 0xFFFFFFFF: the default, about 4 M polls).  A wait that gives up records
 * SEVP_TIMEOUT for sevp_nn_tc_status, skips the stores and returns after
 * draining (with the default limit) the copies and MMAs already issued.
 * Process-wide; synchronises the device. */
int sevp_nn_tc_set_wait_limit(unsigned limit);

/* Weight gradient of the 3x3 convolution, FP32, accumulated into dw
 * [9][cin][cout] (and db [cout] when given); dy is masked like the data
 * gradient when mask is given. */
int sevp_nn_conv3x3_wgrad(const void *x, int x_ld, int x_off, int cin, const void *dy, int dy_ld,
                          int dy_off, int cout, const void *mask, int mask_ld, int mask_off,
                          float *dw, float *db, int B, int H, int W, void *stream);

/* Weight gradient of the 3x3 convolution on the tcgen05 tensor cores (FP32
 * accumulator in tensor memory), accumulated into dw [9][cin][cout]:
 *   dw[tap][ci][co] += sum_p x[p + shift(tap)][x_off + ci] * g[p][co]
 * with g the packed output gradient [B*H*W][cout] (ReLU mask already
 * applied).  cin and cout multiples of 16 up to 256; x_ld, x_off multiples
 * of 8; x and g 16-byte aligned.  The same sums as sevp_nn_conv3x3_wgrad up
 * to the FP32 summation order. */
int sevp_nn_conv3x3_wgrad_tc(const void *x, int x_ld, int x_off, int cin, const void *g, int cout,
                             float *dw, int B, int H, int W, void *stream);
/* The whole backward of one 3x3 convolution + ReLU on the tensor cores:
 * packs dy masked by mask > 0 into scratch (B*H*W*cout BF16), then the
 * weight gradient (sevp_nn_conv3x3_wgrad_tc, into dw), the bias gradient
 * (into db when given) and, when dx is given, the data gradient
 * (sevp_nn_conv3x3_tma with the mirrored weights wm, written to dx). */
int sevp_nn_conv3x3_backward_tc(const void *x, int x_ld, int x_off, int cin, const void *dy,
                                int dy_ld, int dy_off, int cout, const void *mask, int mask_ld,
                                int mask_off, const void *wm, void *scratch, float *dw, float *db,
                                void *dx, int dx_ld, int dx_off, int B, int H, int W,
                                void *stream);

/* wt[tap][co][ci] = w[tap][ci][co] (BF16). */
int sevp_nn_weight_transpose(const void *w, void *wt, int cin, int cout, void *stream);
/* wm[tap][ci][co] = w[8 - tap][ci][co] (BF16): the K-major weights of the
 * data gradient as a forward convolution from cout to cin channels. */
int sevp_nn_weight_mirror(const void *w, void *wm, int cin, int cout, void *stream);
/* Data gradient of the 3x3 convolution on the tcgen05 tensor cores:
 *   dx[p][dx_off + ci] = sum_{tap, co} dy'[p + shift(tap)][co] * wm[tap][ci][co]
 * with dy' = dy where mask > 0 (the ReLU of the forward output; all of dy
 * when mask is NULL), packed into scratch (B*H*W*cout BF16, 16-byte
 * aligned) and convolved by sevp_nn_conv3x3_tma with the mirrored weights
 * of sevp_nn_weight_mirror.  The same result as sevp_nn_conv3x3 with flip
 * = 1 up to the FP32 summation order; limits of sevp_nn_conv3x3_tma, with
 * cout as its input channels. */
int sevp_nn_conv3x3_dgrad_tc(const void *dy, int dy_ld, int dy_off, int cout, const void *mask,
                             int mask_ld, int mask_off, const void *wm, void *scratch, void *dx,
                             int dx_ld, int dx_off, int cin, int B, int H, int W, void *stream);

/* 2x2 average pooling of C channels (H, W even): forward H x W -> H/2 x W/2;
 * backward spreads a quarter of each gradient to its four inputs (added to
 * out when accumulate != 0). */
int sevp_nn_pool(const void *in, int in_ld, int in_off, void *out, int out_ld, int out_off, int C,
                 int B, int H, int W, int backward, int accumulate, void *stream);

/* Nearest 2x upsampling (H, W are the output size): forward H/2 x W/2 ->
 * H x W; backward sums each 2x2 block of gradients. */
int sevp_nn_upsample(const void *in, int in_ld, int in_off, void *out, int out_ld, int out_off,
                     int C, int B, int H, int W, int backward, void *stream);

/* 1x1 FP32 head, C -> 1 channel: forward y[p] = b + sum_c x[p][c] w[c];
 * backward (backward != 0) dx = dy w^T (BF16) and dw, db (FP32, summed). */
int sevp_nn_head(const void *x, int x_ld, int x_off, int C, const float *w, const float *b,
                 float *y, const float *dy, void *dx, int dx_ld, int dx_off, float *dw, float *db,
                 long long P, int backward, void *stream);

/* Mean squared error: loss += inv_n * sum (valid (y - t))^2 and
 * dy = 2 inv_n valid (y - t) (valid optional: all ones). */
int sevp_nn_mse(const float *y, const float *t, const float *valid, float *dy, float *loss,
                long long P, float inv_n, void *stream);

/* One Adam step on FP32 master weights w (gradient g, moments m, v; L2
 * weight decay wd added to the gradient; bias corrections for `step`);
 * refreshes the BF16 copy w16 and/or an FP32 copy w32 when given. */
int sevp_nn_adam(float *w, const float *g, float *m, float *v, void *w16, float *w32, long long n,
                 float lr, float b1, float b2, float eps, int step, float wd, void *stream);

/* b = BF16(a). */
int sevp_nn_to_bf16(const float *a, void *b, long long n, void *stream);

/* Warm-start features of a solver context (on its stream):
 *   e = 2 eta1 - eta2, m = M^-1 (b - A e) (one tile-SEVP solve), d = eta1 - eta2,
 * the three fields averaged over coarse x coarse cells (coarse 1, 2, 4, 8 or
 * 16 dividing nx and ny), scales = the RMS of those averages over the cells,
 * and feat = the averages divided by their scales, as BF16 channels 0..2 of
 * 16 on a wn x hn grid (multiples of 8, at least nx/coarse x ny/coarse;
 * zero padding). */
int sevp_nn_features(sevp_ctx *ctx, const double *eta1, const double *eta2, const double *b,
                     double *e, double *m, double *d, void *feat, float *scales, int coarse,
                     int wn, int hn);

/* Training target t = (eta - e - m) / scales[1] on the network grid
 * (coarse-cell averages, zero on the padding). */
int sevp_nn_target(sevp_ctx *ctx, const double *eta, const double *e, const double *m,
                   const float *scales, float *t, int coarse, int wn, int hn);

/* Guess x = e + m + scales[1] * y, y interpolated bilinearly between network
 * cell centres when coarse > 1. */
int sevp_nn_combine(sevp_ctx *ctx, const double *e, const double *m, const float *y,
                    const float *scales, double *x, int coarse, int wn, int hn);

/* The context's CUDA stream, and a counter of kernels launched on behalf of
 * the context by a caller (added to sevp_kernel_launches). */
void *sevp_stream(const sevp_ctx *ctx);
int sevp_add_launches(sevp_ctx *ctx, int n);

#ifdef __cplusplus
}
#endif

#endif /* SEVP_NN_H */
