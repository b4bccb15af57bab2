/* Kernels of the learned history warm start (orthoroute_b200/warm.py).
 *
 * No counterpart in the reference: OrthoRoute starts every route from zero
 * history.  These entry points run a small 3D convolutional net that predicts
 * the converged history field of a board from its pins and airwires, and train
 * it.  Activations are bf16 tensors laid out [D][H][W][C] (channels last),
 * weights fp32 masters [27][Cin][Cout] packed to bf16 for the convolution,
 * all device pointers; every call returns an ORSP status and runs on `stream`.
 */
#ifndef ORSP_WARM_H
#define ORSP_WARM_H

#include "orsp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* 3x3x3 convolution with zero padding, bias and optional ReLU on the tensor
 * cores (bf16 in, fp32 accumulate): Y[v][co] = act(bias[co] + sum over taps
 * and ci of Xm[v+tap][ci] * Wt[tap][ci][co]).  Xm = X, or X where mask > 0
 * and 0 elsewhere when mask (same layout as X) is given - the ReLU derivative
 * of a layer output applied to its incoming gradient.  Output to Y (bf16) or,
 * when Yf is given, to Yf (fp32).  Cin and Cout multiples of 16, Cout <= 64. */
ORSP_API int orsp_warm_conv3d(const void *X, const void *mask, const void *Wt, const float *bias, void *Y,
                              float *Yf, int32_t D, int32_t H, int32_t W, int32_t Cin, int32_t Cout,
                              int32_t relu, uintptr_t stream);

/* The same convolution (same arguments and results up to the summation
 * order of the fp32 accumulation) on the 5th-generation tensor cores:
 * tcgen05.mma with bf16 operands staged in shared memory in the canonical
 * K-major layout and the fp32 accumulator in tensor memory (128 voxels x
 * Cout per tile), persistent CTAs.  Cin and Cout multiples of 16, Cout <= 64,
 * and all 27 x Cin x Cout weights within shared memory (Cin x Cout <= 2048
 * for Cout <= 32; Cin <= 32 for Cout = 64).  A wait that expires (2 s) is
 * recorded for orsp_warm_tc_status. */
ORSP_API int orsp_warm_conv3d_tc(const void *X, const void *mask, const void *Wt, const float *bias, void *Y,
                                 float *Yf, int32_t D, int32_t H, int32_t W, int32_t Cin, int32_t Cout,
                                 int32_t relu, uintptr_t stream);

/* The weight and bias gradients of orsp_warm_wgrad on the tensor cores
 * (tcgen05.mma, both operands MN-major, one TMEM accumulator per group of
 * 128 / Cin taps, partial sums added to dW with fp32 atomics).  Cin, Cout
 * multiples of 16, at most 64, with ceil(27 Cin / 128) x Cout <= 512
 * accumulator columns. */
ORSP_API int orsp_warm_wgrad_tc(const void *X, const void *dY, const void *Yo, float *dW, float *db, int32_t D,
                                int32_t H, int32_t W, int32_t Cin, int32_t Cout, uintptr_t stream);

/* 1 in *expired if a tensor-core convolution gave up on a wait since the
 * last call (then its output is incomplete), else 0; clears the record.
 * Synchronises with the device. */
ORSP_API int orsp_warm_tc_status(int32_t *expired);

/* Weight and bias gradients of a convolution: dW[tap][ci][co] +=
 * sum_v X[v+tap][ci] * G[v][co] and db[co] += sum_v G[v][co] (db optional),
 * with G = dY, or dY where Yo > 0 when the layer's ReLU output Yo is given.
 * dW, db are fp32 and accumulated into.  Cin, Cout multiples of 16, <= 64. */
ORSP_API int orsp_warm_wgrad(const void *X, const void *dY, const void *Yo, float *dW, float *db, int32_t D,
                             int32_t H, int32_t W, int32_t Cin, int32_t Cout, uintptr_t stream);

/* 2x2 average pooling in x and y: Y [D][H/2][W/2][C] from X [D][H][W][C]. */
ORSP_API int orsp_warm_pool(const void *X, void *Y, int32_t D, int32_t H, int32_t W, int32_t C, uintptr_t stream);

/* Fine [D][H][W][C] from coarse [D][H/2][W/2][C]: Xf = scale * Yc of the
 * covering coarse cell (nearest upsampling with scale 1, the adjoint of the
 * pooling with scale 0.25). */
ORSP_API int orsp_warm_spread(const void *Yc, void *Xf, int32_t D, int32_t H, int32_t W, int32_t C, float scale,
                              uintptr_t stream);

/* Coarse [D][H/2][W/2][C] = sum of the four covering fine cells (the adjoint
 * of nearest upsampling). */
ORSP_API int orsp_warm_gather4(const void *Xf, void *Yc, int32_t D, int32_t H, int32_t W, int32_t C,
                               uintptr_t stream);

/* out = a + b over n bf16 values. */
ORSP_API int orsp_warm_add(const void *a, const void *b, void *out, int64_t n, uintptr_t stream);

/* Mean squared error of the first `used` channels of P (fp32 [nvox][C])
 * against T (fp32 [nvox][used]), per-voxel weights wv (optional):
 * loss[0] += inv_count * sum w (p - t)^2, dP (bf16 [nvox][C]) = 2 w (p - t)
 * inv_count on the used channels, 0 on the others. */
ORSP_API int orsp_warm_mse(const float *P, const float *T, const float *wv, void *dP, float *loss, int64_t nvox,
                           int32_t C, int32_t used, float inv_count, uintptr_t stream);

/* One Adam step on n fp32 values (lr_t includes the bias corrections; wd is
 * L2 weight decay added to the gradient). */
ORSP_API int orsp_warm_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr_t, float b1,
                            float b2, float eps, float wd, uintptr_t stream);

/* bf16 weights for orsp_warm_conv3d from fp32 w [27][Cin][Cout]: as is
 * (transpose = 0) or, for the gradient with respect to the input, taps
 * mirrored and channels swapped, Wt[tap][co][ci] = w[26 - tap][ci][co]. */
ORSP_API int orsp_warm_pack_weights(const float *w, void *Wt, int32_t Cin, int32_t Cout, int32_t transpose,
                                    uintptr_t stream);

#ifdef __cplusplus
}
#endif

#endif /* ORSP_WARM_H */
