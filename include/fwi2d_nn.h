/*
 * fwi2d_nn.h — kernels of the CNN gradient preconditioner (libfwi2d.so).
 *
 * No reference counterpart: the reference's FWI uses the illumination-
 * normalised gradient only (inversion.cu:111-166, 286-358).  These entry
 * points let a host driver run a U-Net between fwi_gradient_accumulate and
 * the line search, and train it, on device buffers it owns:
 *   - activations: NHWC bfloat16 (uint16 storage), channels a multiple of 16;
 *   - activation gradients, master weights, optimiser state: float32;
 *   - weights: [Cout][3][3][Cin], biases: [Cout];
 *   - every call enqueues on `stream` (a cudaStream_t, NULL = default) and
 *     returns 0, or FWI_ERR_ARG for unsupported sizes;
 *   - buffers start on 16-byte boundaries and channel counts (and relu_bwd's
 *     n) are multiples of 8: the kernels move 8 channels at a time.
 * The 3x3 convolutions (zero padding) are implicit GEMMs on the BF16 tensor
 * cores with FP32 accumulation.
 */
#ifndef FWI2D_NN_H
#define FWI2D_NN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* out[p, co] = act(bias[co] + sum_{tap, ci} in[p + tap, ci] w[co, tap, ci]);
 * act = ReLU when relu != 0.  out_bf16 and/or out_f32 ([N,H,W,Cout]) may be
 * NULL; bias may be NULL.  Cin, Cout multiples of 16, at most 256.  The data
 * gradient of a convolution is this call on the output gradient with wt of
 * fwi_nn_weight_prep, Cin and Cout swapped.  Runs on the tcgen05 tensor cores
 * with the accumulator in tensor memory; fwi_nn_conv3x3_mma computes the same
 * on the mma.sync path (the first implementation, kept for comparison). */
int fwi_nn_conv3x3(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout,
                   int relu, void* out_bf16, float* out_f32, void* stream);
int fwi_nn_conv3x3_mma(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout,
                       int relu, void* out_bf16, float* out_f32, void* stream);
/* Synchronises the device; FWI_ERR_TIMEOUT when a bounded wait inside a
 * tcgen05 convolution gave up since the last call (the flag is then reset). */
int fwi_nn_check(void);
/* dw[co, tap, ci] = sum_p dout[p, co] in[p + tap, ci]; db[co] = sum_p dout[p, co]
 * (db may be NULL).  partial: fwi_nn_wgrad_partial_floats(...) floats of
 * scratch; the sums are in a fixed order (deterministic). */
size_t fwi_nn_wgrad_partial_floats(int N, int H, int W, int Cin, int Cout);
int fwi_nn_conv3x3_wgrad(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, float* partial,
                         float* dw, float* db, void* stream);
/* The per-chunk sums run on the tcgen05 tensor cores for Cout <= 128 (M =
 * output channels padded to 128, N = several taps x input channels, K =
 * pixels, both operands MN-major; the bias gradient as one more MMA against
 * ones), else on mma.sync; _mma always uses mma.sync (for comparison). */
int fwi_nn_conv3x3_wgrad_mma(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, float* partial,
                             float* dw, float* db, void* stream);
/* bf16 copy of float32 weights w and (wt != NULL) the data-gradient weights
 * wt[ci][8 - tap][co]. */
int fwi_nn_weight_prep(const float* w, int Cout, int Cin, void* w_bf16, void* wt_bf16, void* stream);
/* 2x2 average pooling to (H/2, W/2) and its gradient (accumulate != 0: +=). */
int fwi_nn_pool2(const void* in, int N, int H, int W, int C, void* out, void* stream);
int fwi_nn_pool2_bwd(const float* dout, int N, int H, int W, int C, float* din, int accumulate, void* stream);
/* out = concat(nearest 2x upsampling of a (N,Hs,Ws,C1) onto (H,W), skip (N,H,W,C2))
 * and its gradient split into da and dskip. */
int fwi_nn_upcat(const void* a, int Hs, int Ws, int C1, const void* skip, int N, int H, int W, int C2, void* out,
                 void* stream);
int fwi_nn_upcat_bwd(const float* dout, int N, int H, int W, int C1, int C2, int Hs, int Ws, float* da, int acc_a,
                     float* dskip, int acc_skip, void* stream);
/* dpre = da * (a > 0) in bf16. */
int fwi_nn_relu_bwd(const float* da, const void* a, size_t n, void* dpre, void* stream);
/* loss = sum_p (mask_p (out_f32[p, 0] - target[p]))^2 (FP64); dout[p, 0] =
 * 2 mask_p (out - target) scale, other channels 0.  partial: 256 doubles. */
int fwi_nn_mse(const float* out_f32, int C, const float* target, const float* mask, long long P, float scale,
               void* dout, double* partial, double* loss, void* stream);
/* Adam step `step` (1-based) on float32 weights. */
int fwi_nn_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float beta1, float beta2, float eps,
                int step, void* stream);
/* Network input from the raw gradient g, the illumination il and the velocity
 * v (nz x nx float32, z fastest): NHWC bf16 with H = nx, W = nz, C = 16:
 *   ch0 = q / max|q|, q = g / (il + 1e-3 max il)
 *   ch1 = 1 + log10(il / max il + 1e-6) / 6
 *   ch2 = (v - v0) vs,  ch3..15 = 0.
 * scratch: 2 device words. */
int fwi_nn_pack_inputs(const float* g, const float* il, const float* v, int nz, int nx, float v0, float vs,
                       unsigned* scratch, void* out, void* stream);
/* dst[p] = out_f32[p, 0]. */
int fwi_nn_unpack(const float* out_f32, int C, long long P, float* dst, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FWI2D_NN_H */
