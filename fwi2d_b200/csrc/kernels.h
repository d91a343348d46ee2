// kernels.h — launch wrappers of the device kernels (all enqueue on `st`).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "kargs.h"

namespace fwi {

// ---- k_stencil.cu ------------------------------------------------------------
dim3 step_grid(int ldz, int max_nxx, int nshots);
void launch_fwd_step(const FwdArgs& a, dim3 grid, cudaStream_t st);
void launch_bwd_step(const BwdArgs& a, bool gradient, dim3 grid, cudaStream_t st);

// ---- k_fwd_tma.cu --------------------------------------------------------------
int fwd_tma_rows();                                   // rows per tile (128)
bool fwd_tma_supported(const FwdTmaConfig& c);
size_t fwd_tma_smem(const FwdTmaConfig& c);           // dynamic shared memory bytes
int fwd_tma_box_cur_z(const FwdTmaConfig& c);
int fwd_tma_box_cur_x(const FwdTmaConfig& c);
int fwd_tma_box_pt_z(const FwdTmaConfig& c);
int fwd_tma_box_pt_x(const FwdTmaConfig& c);
cudaError_t fwd_tma_configure(int* ctas_per_sm_out, const FwdTmaConfig& c);
cudaError_t launch_fwd_tma(const FwdTmaConfig& c, const CUtensorMap& m_cur, const CUtensorMap& m_old,
                           const CUtensorMap& m_vel, const FwdTmaArgs& a, int grid, cudaStream_t st);

// ---- k_fwd_loop.cu -------------------------------------------------------------
// Tensor maps of the four field buffers (Q^t box with a 4-cell halo, pointwise
// box) and of the velocity, passed by value to the cooperative kernel.
struct FwdLoopMaps {
    CUtensorMap cur[4];
    CUtensorMap pt[4];
    CUtensorMap vel;
};
// TX tile columns, S pipeline stages, B CTAs per SM the registers are budgeted for
bool fwd_loop_supported(int TX, int S, int B);
cudaError_t fwd_loop_configure(int* ctas_per_sm, int TX, int S, int B);
cudaError_t launch_fwd_loop(int TX, int S, int B, const FwdLoopMaps& maps, const FwdLoopArgs& la, int grid,
                            cudaStream_t st);

// ---- k_fwd_res.cu --------------------------------------------------------------
int fwd_res_threads();               // compute threads per CTA
int fwd_res_max_rec();               // receiver entries per slab
int fwd_res_max_src();               // injection points per slab
bool fwd_res_fits(int w, int ldz);   // a slab of w columns fits the kernel's item and halo tables
size_t fwd_res_smem(int wmax, int ldz);  // dynamic shared memory for slabs up to wmax columns
size_t fwd_res_stage_smem(int ldz);      // of which the halo staging
size_t fwd_res_static_smem();
cudaError_t fwd_res_configure(int ldz, size_t smem, int* ctas_per_sm);
cudaError_t launch_fwd_res(const FwdResArgs& a, size_t smem, cudaStream_t st);

// ---- k_bwd_loop.cu -------------------------------------------------------------
// Tensor maps of the backward kernel: stencil boxes (128+8 rows, TX+8 columns)
// and pointwise boxes (128 rows, TX columns), indexed like BwdLoopArgs.ps/pr.
struct BwdLoopMaps {
    CUtensorMap ps_st[2], pr_st[2];  // [p]: the buffer read through the stencil at parity p
    CUtensorMap ps_pt[2], pr_pt[2];  // [p]: the buffer read and written pointwise at parity p
    CUtensorMap acc_a, acc_b, vel;
};
bool bwd_loop_supported(int TX, int S);
cudaError_t bwd_loop_configure(int* ctas_per_sm, int TX, int S);
cudaError_t launch_bwd_loop(int TX, int S, bool gradient, const BwdLoopMaps& maps, const BwdLoopArgs& la, int grid,
                            cudaStream_t st);

// ---- k_rbc.cu ----------------------------------------------------------------
struct BumpDev { float xc, zc, r, A, factor; };
struct RbcArgs {
    const float* base;         // edge-replicated velocity, padded layout
    long long base_stride;     // per-shot stride of base (0: shared)
    float* out;                // random-boundary velocity per shot
    long long out_stride;
    const int* nxx;            // per-shot padded width
    const int* shot_id;        // survey index of each shot (RNG stream)
    const BumpDev* bumps;
    const int* bump_ptr;       // per shot: bumps[bump_ptr[s] .. bump_ptr[s+1])
    int nzz, ldz, nb, max_nxx;
    float dh, varVp, vmin, vmax;
    uint64_t seed;
};
void launch_rbc(const RbcArgs& a, int nshots, cudaStream_t st);

// ---- k_util.cu ---------------------------------------------------------------
// padded(i,j) = model(clamp(i-nb), c0 + clamp(j-nb, 0, w-1)), nz x nx model,
// one window per shot (c0[s], w[s]); rows nzz..ldz-1 are zeroed.
void launch_expand(const float* model, int nz, int nx, float* out, long long out_stride, const int* c0,
                   const int* w, int nshots, int nb, int nzz, int ldz, int max_nxx, cudaStream_t st);
// out(i,x) (+)= sum over the shots s whose window [c0[s], c0[s]+w[s]) holds
// column x of padded_s(i+nb, x-c0[s]+nb); nz x nx.  Fixed shot order.
void launch_crop_sum(const float* padded, long long stride, int nshots, int nb, int ldz, int nz, int nx,
                     const int* c0, const int* w, float* out, bool accumulate, cudaStream_t st);
// Zeroes the nt samples of every trace whose keep[] entry is 0.
void launch_mask_traces(float* data, const unsigned char* keep, size_t ntraces, int nt, cudaStream_t st);
// RTM post-processing (migration.cu:90-115): q = img/illum, out = -d2q/dz2 * idh2.
void launch_rtm_post(const float* img, const float* illum, int nz, int nx, float idh2, float* out, cudaStream_t st);
// Gradient post-processing (inversion.cu:136-165) without the final scaling:
// q = g/illum, out = -d2q/dz2 * idh2 below row zmask_i, |out| max into *gmax_bits.
void launch_grad_post(const float* g, const float* illum, int nz, int nx, float idh2, int zmask_i, float* out,
                      unsigned int* gmax_bits, cudaStream_t st);
void launch_scale_by_inverse(float* x, size_t n, const unsigned int* gmax_bits, cudaStream_t st);
// *bits = float bits of max |x| (order-independent, deterministic)
void launch_absmax(const float* x, size_t n, unsigned int* bits, cudaStream_t st);
// res = obs - cal over n samples, per-block FP64 partial sums of res^2 into
// partial[], then a fixed-order sum into *out.  Deterministic.
int  residual_blocks(size_t n);
void launch_residual(const float* obs, const float* cal, float* res, size_t n, double* partial, double* out,
                     cudaStream_t st);
// vp = 1/sqrtf(m - alpha*g)  (inversion.cu:312-317)
void launch_trial_velocity(const float* m, const float* g, float alpha, float* vp, size_t n, cudaStream_t st);
// m -= step*g; vp = 1/sqrtf(m)  (inversion.cu:346-352)
// with mlo > 0 the new slowness^2 is clamped to [mlo, mhi]
void launch_update_model(float* m, const float* g, float step, float* vp, size_t n, cudaStream_t st,
                         float mlo = 0.0f, float mhi = 0.0f);
// m = 1/(vp*vp)  (inversion.cu:101-109)
void launch_slowness2(const float* vp, float* m, size_t n, cudaStream_t st);
// Sets *flag to 1 when any of x[0..n) is not finite.
void launch_check_finite(const float* x, size_t n, int* flag, cudaStream_t st);
// Adds scale*series[soff[k] + sample] at the listed points of each shot
// (the injection of time level 0, before the first step).
void launch_inject_points(float* field, long long fstride, const ShotDesc* shots, int nshots, InjTable inj,
                          int ldz, cudaStream_t st);

// ---- k_prep.cu -------------------------------------------------------------------
// Direct-wave mute of nsrc seismograms (nrec x nt trace-major each) in place;
// bits: nsrc scratch words.  Geometry arrays are on the device.
void launch_mute_direct(float* data, int nsrc, int nrec, int nt, const float* sx, const float* sz, const float* rx,
                        const float* rz, float velocity, float delay, float dt, float gstd, unsigned* bits,
                        cudaStream_t st);
// out = 1 / G(1 / vp) below row keep_rows, vp above; weights[0..radius] the
// half of the normalised Gaussian; tmp: nz*nx scratch.
void launch_smooth_slowness(const float* vp, int nz, int nx, const double* weights, int radius, int keep_rows,
                            float* tmp, float* out, cudaStream_t st);

// ---- k_nn.cu (CNN preconditioner; bf16 buffers passed as void*) ----------------
// TMA-fed, warp-specialised tcgen05 kernels (k_nn_tma.cu): the convolution
// (Cin, Cout multiples of 16, <= 256) and the weight-gradient chunk partials
// (Cout <= 128; returns the number of chunks, -1 for unsupported sizes);
// partial holds [chunk][co][tap][ci] then, when bias, [chunk][co];
// nn_tma_error: 1 when a bounded wait of either kernel gave up since the last reset
int  nn_conv3x3_tma(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout,
                    int relu, void* out, float* out32, cudaStream_t st);
size_t nn_wgrad_tma_partial_floats(int N, int H, int W, int Cin, int Cout);
int  nn_wgrad_tma(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, float* partial, bool bias,
                  cudaStream_t st);
int  nn_tma_error(bool reset);
// mma.sync m16n8k16 implicit GEMM (k_nn.cu)
int  nn_conv3x3_mma(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout,
                    int relu, void* out, float* out32, cudaStream_t st);
int  nn_wgrad_chunks(long long P);
// tensor_memory: chunk partials on the tcgen05 kernel (Cout <= 128), else mma.sync
int  nn_conv3x3_wgrad(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, float* partial,
                      float* dw, float* db, cudaStream_t st, bool tensor_memory = true);
void nn_weight_prep(const float* w, int Cout, int Cin, void* wb, void* wt, cudaStream_t st);
void nn_pool_fwd(const void* in, int N, int H, int W, int C, void* out, cudaStream_t st);
void nn_pool_bwd(const float* dout, int N, int H, int W, int C, float* din, int accumulate, cudaStream_t st);
void nn_upcat_fwd(const void* a, int Hs, int Ws, int C1, const void* skip, int N, int H, int W, int C2, void* out,
                  cudaStream_t st);
void nn_upcat_bwd(const float* dout, int N, int H, int W, int C1, int C2, int Hs, int Ws, float* da, int acc_a,
                  float* dskip, int acc_skip, cudaStream_t st);
void nn_relu_bwd(const float* da, const void* a, size_t n, void* dpre, cudaStream_t st);
void nn_mse(const float* out32, int C, const float* target, const float* mask, long long P, float scale, void* dout,
            double* partial, double* loss, cudaStream_t st);
void nn_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps, int step,
             cudaStream_t st);
void nn_pack_inputs(const float* g, const float* il, const float* v, int nz, int nx, float v0, float vs,
                    unsigned* bits, void* out, cudaStream_t st);
void nn_unpack_channel(const float* out32, int C, long long P, float* dst, cudaStream_t st);

// ---- k_noalloc.cu --------------------------------------------------------------
size_t noalloc_max_samples();
int residual_noalloc(const float* d_obs, const float* d_cal, float* d_res, size_t n, double* d_sum,
                     cudaStream_t st, std::string* err);

}  // namespace fwi
