// capi_nn.cpp — extern "C" surface of fwi2d_nn.h over the kernels of k_nn.cu.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fwi2d.h"
#include "../../include/fwi2d_nn.h"
#include "kernels.h"

namespace {
cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }
int status() { return cudaGetLastError() == cudaSuccess ? FWI_OK : FWI_ERR_CUDA; }
bool dims_ok(int N, int H, int W) { return N >= 1 && H >= 1 && W >= 1; }
// the element-wise kernels move 8 channels (16 or 32 bytes) at a time
bool vec_ok(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
}  // namespace

extern "C" {

int fwi_nn_conv3x3(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout,
                   int relu, void* out_bf16, float* out_f32, void* stream) {
    if (!in || !w || (!out_bf16 && !out_f32) || !dims_ok(N, H, W)) return FWI_ERR_ARG;
    const int rc = fwi::nn_conv3x3_tma(in, N, H, W, Cin, w, bias, Cout, relu, out_bf16, out_f32, S(stream));
    if (rc == -1) return FWI_ERR_ARG;
    if (rc != 0) return FWI_ERR_CUDA;
    return status();
}

int fwi_nn_conv3x3_mma(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout,
                       int relu, void* out_bf16, float* out_f32, void* stream) {
    if (!in || !w || (!out_bf16 && !out_f32) || !dims_ok(N, H, W)) return FWI_ERR_ARG;
    if (fwi::nn_conv3x3_mma(in, N, H, W, Cin, w, bias, Cout, relu, out_bf16, out_f32, S(stream)) != 0)
        return FWI_ERR_ARG;
    return status();
}

int fwi_nn_check(void) {
    if (cudaDeviceSynchronize() != cudaSuccess) return FWI_ERR_CUDA;
    const int e = fwi::nn_tma_error(true);
    if (e < 0) return FWI_ERR_CUDA;
    return e ? FWI_ERR_TIMEOUT : FWI_OK;
}

size_t fwi_nn_wgrad_partial_floats(int N, int H, int W, int Cin, int Cout) {
    // the larger of the mma.sync path's [chunk][co][tap][ci] and the tcgen05
    // path's, which adds the [chunk][co] bias partials
    const size_t mma = (size_t)fwi::nn_wgrad_chunks((long long)N * H * W) * (size_t)Cout * 9 * Cin;
    const size_t tc = fwi::nn_wgrad_tma_partial_floats(N, H, W, Cin, Cout);
    return mma > tc ? mma : tc;
}

int fwi_nn_conv3x3_wgrad(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, float* partial,
                         float* dw, float* db, void* stream) {
    if (!in || !dout || !partial || !dw || !dims_ok(N, H, W)) return FWI_ERR_ARG;
    const int rc = fwi::nn_conv3x3_wgrad(in, dout, N, H, W, Cin, Cout, partial, dw, db, S(stream), true);
    if (rc == -1) return FWI_ERR_ARG;
    if (rc != 0) return FWI_ERR_CUDA;
    return status();
}

int fwi_nn_conv3x3_wgrad_mma(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, float* partial,
                             float* dw, float* db, void* stream) {
    if (!in || !dout || !partial || !dw || !dims_ok(N, H, W)) return FWI_ERR_ARG;
    if (fwi::nn_conv3x3_wgrad(in, dout, N, H, W, Cin, Cout, partial, dw, db, S(stream), false) != 0)
        return FWI_ERR_ARG;
    return status();
}

int fwi_nn_weight_prep(const float* w, int Cout, int Cin, void* w_bf16, void* wt_bf16, void* stream) {
    if (!w || !w_bf16 || Cout < 1 || Cin < 1) return FWI_ERR_ARG;
    fwi::nn_weight_prep(w, Cout, Cin, w_bf16, wt_bf16, S(stream));
    return status();
}

int fwi_nn_pool2(const void* in, int N, int H, int W, int C, void* out, void* stream) {
    if (!in || !out || !dims_ok(N, H / 2, W / 2) || C < 1 || C % 8 || !vec_ok(in) || !vec_ok(out)) return FWI_ERR_ARG;
    fwi::nn_pool_fwd(in, N, H, W, C, out, S(stream));
    return status();
}

int fwi_nn_pool2_bwd(const float* dout, int N, int H, int W, int C, float* din, int accumulate, void* stream) {
    if (!dout || !din || !dims_ok(N, H / 2, W / 2) || C < 1 || C % 8 || !vec_ok(dout) || !vec_ok(din))
        return FWI_ERR_ARG;
    fwi::nn_pool_bwd(dout, N, H, W, C, din, accumulate, S(stream));
    return status();
}

int fwi_nn_upcat(const void* a, int Hs, int Ws, int C1, const void* skip, int N, int H, int W, int C2, void* out,
                 void* stream) {
    if (!a || !skip || !out || !dims_ok(N, H, W) || Hs < 1 || Ws < 1 || C1 < 1 || C2 < 1 || C1 % 8 || C2 % 8 ||
        !vec_ok(a) || !vec_ok(skip) || !vec_ok(out))
        return FWI_ERR_ARG;
    fwi::nn_upcat_fwd(a, Hs, Ws, C1, skip, N, H, W, C2, out, S(stream));
    return status();
}

int fwi_nn_upcat_bwd(const float* dout, int N, int H, int W, int C1, int C2, int Hs, int Ws, float* da, int acc_a,
                     float* dskip, int acc_skip, void* stream) {
    if (!dout || !da || !dskip || !dims_ok(N, H, W) || Hs < 1 || Ws < 1 || C1 < 8 || C2 < 8 || C1 % 8 || C2 % 8 ||
        !vec_ok(dout) || !vec_ok(da) || !vec_ok(dskip))
        return FWI_ERR_ARG;
    fwi::nn_upcat_bwd(dout, N, H, W, C1, C2, Hs, Ws, da, acc_a, dskip, acc_skip, S(stream));
    return status();
}

int fwi_nn_relu_bwd(const float* da, const void* a, size_t n, void* dpre, void* stream) {
    if (!da || !a || !dpre || n % 8 || !vec_ok(da) || !vec_ok(a) || !vec_ok(dpre)) return FWI_ERR_ARG;
    fwi::nn_relu_bwd(da, a, n, dpre, S(stream));
    return status();
}

int fwi_nn_mse(const float* out_f32, int C, const float* target, const float* mask, long long P, float scale,
               void* dout, double* partial, double* loss, void* stream) {
    if (!out_f32 || !target || !dout || !partial || !loss || C < 8 || C % 8 || P < 1 || !vec_ok(dout))
        return FWI_ERR_ARG;
    fwi::nn_mse(out_f32, C, target, mask, P, scale, dout, partial, loss, S(stream));
    return status();
}

int fwi_nn_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float beta1, float beta2, float eps,
                int step, void* stream) {
    if (!w || !g || !m || !v || step < 1) return FWI_ERR_ARG;
    fwi::nn_adam(w, g, m, v, n, lr, beta1, beta2, eps, step, S(stream));
    return status();
}

int fwi_nn_pack_inputs(const float* g, const float* il, const float* v, int nz, int nx, float v0, float vs,
                       unsigned* scratch, void* out, void* stream) {
    if (!g || !il || !v || !scratch || !out || nz < 1 || nx < 1) return FWI_ERR_ARG;
    fwi::nn_pack_inputs(g, il, v, nz, nx, v0, vs, scratch, out, S(stream));
    return status();
}

int fwi_nn_unpack(const float* out_f32, int C, long long P, float* dst, void* stream) {
    if (!out_f32 || !dst || C < 1 || P < 1) return FWI_ERR_ARG;
    fwi::nn_unpack_channel(out_f32, C, P, dst, S(stream));
    return status();
}

}  // extern "C"
