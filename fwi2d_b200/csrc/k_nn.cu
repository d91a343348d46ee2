// k_nn.cu — kernels of the CNN gradient preconditioner (a 4-level U-Net on
// the FWI gradient, illumination and model; no reference counterpart).
//
// Activations are NHWC bfloat16 (channels innermost, a multiple of 16);
// gradients of activations are float32.  The convolutions the network runs
// are the tcgen05 kernels of k_nn_tma.cu; this file holds the element-wise
// layers, the fixed-order reductions, Adam, and the first implementation of
// the convolutions on the warp-level tensor-core path (mma.sync m16n8k16,
// fwi_nn_conv3x3_mma / _wgrad_mma, kept for comparison), implicit GEMMs with
// FP32 accumulation:
//   forward   out[p, co] = sum_{tap, ci} in[p + tap, ci] * w[co, tap, ci]
//   data grad the same kernel on the output gradient with the flipped,
//             transposed weights wT[ci, 8 - tap, co]
//   weight grad dW[co, tap, ci] = sum_p dout[p, co] * in[p + tap, ci], pixels
//             split over CTAs into per-chunk partials summed in a fixed order
// (zero padding at the image border).  A warp owns 16 consecutive pixels of
// one image row and NT x 8 output channels.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace fwi {

namespace {

__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16* p) {
    return __ldg(reinterpret_cast<const unsigned int*>(p));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int kWarps = 4;  // warps per CTA, each on its own 16-pixel run

// in: [N,H,W,Cin] bf16; w: [Cout,9,Cin] bf16; out (optional): [N,H,W,Cout]
// bf16 after bias / ReLU; out32 (optional): the same in float32.
template <int NT>
__global__ void __launch_bounds__(32 * kWarps) conv3x3_kernel(const __nv_bfloat16* __restrict__ in, int N, int H,
                                                              int W, int Cin, const __nv_bfloat16* __restrict__ w,
                                                              const float* __restrict__ bias, int Cout, int relu,
                                                              __nv_bfloat16* __restrict__ out,
                                                              float* __restrict__ out32) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int runs = (W + 15) / 16;
    const int x0 = ((blockIdx.x % ((runs + kWarps - 1) / kWarps)) * kWarps + warp) * 16;
    const int y = blockIdx.y;
    const int n = blockIdx.x / ((runs + kWarps - 1) / kWarps);
    const int co0 = blockIdx.z * NT * 8;
    if (x0 >= W || n >= N) return;
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    for (int tap = 0; tap < 9; ++tap) {
        const int yy = y + tap / 3 - 1;
        if (yy < 0 || yy >= H) continue;
        const int xa = x0 + g + tap % 3 - 1, xb = xa + 8;
        const bool oka = xa >= 0 && xa < W, okb = xb >= 0 && xb < W;
        const __nv_bfloat16* rowp = in + ((size_t)n * H + yy) * W * Cin;
        const __nv_bfloat16* pa = rowp + (size_t)(oka ? xa : 0) * Cin + 2 * t;
        const __nv_bfloat16* pb = rowp + (size_t)(okb ? xb : 0) * Cin + 2 * t;
        const __nv_bfloat16* wp = w + ((size_t)(co0 + g) * 9 + tap) * Cin + 2 * t;
        for (int c = 0; c < Cin; c += 16) {
            uint32_t a[4];
            a[0] = oka ? ld_pair(pa + c) : 0u;
            a[1] = okb ? ld_pair(pb + c) : 0u;
            a[2] = oka ? ld_pair(pa + c + 8) : 0u;
            a[3] = okb ? ld_pair(pb + c + 8) : 0u;
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const __nv_bfloat16* wj = wp + (size_t)j * 8 * 9 * Cin + c;
                uint32_t b[2] = {ld_pair(wj), ld_pair(wj + 8)};
                mma_bf16(acc[j], a, b);
            }
        }
    }
    // epilogue: rows g (pixel x0+g) and g+8, columns 2t, 2t+1 of each n8 tile
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int x = x0 + g + 8 * half;
        if (x >= W) continue;
        const size_t p = ((size_t)n * H + y) * W + x;
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int co = co0 + j * 8 + 2 * t;
            float v0 = acc[j][2 * half], v1 = acc[j][2 * half + 1];
            if (bias) {
                v0 += __ldg(bias + co);
                v1 += __ldg(bias + co + 1);
            }
            if (relu) {
                v0 = fmaxf(v0, 0.0f);
                v1 = fmaxf(v1, 0.0f);
            }
            if (out)
                *reinterpret_cast<uint32_t*>(out + p * Cout + co) =
                    pack2(__float2bfloat16_rn(v0), __float2bfloat16_rn(v1));
            if (out32) *reinterpret_cast<float2*>(out32 + p * Cout + co) = make_float2(v0, v1);
        }
    }
}

// Weight gradient partials: CTA (chunk, tap, tile) sums its pixel chunk for
// 16 output channels x NT*8 input channels; warp w takes every kWarps-th
// 16-pixel group of the chunk and the warps are summed in shared memory.
template <int NT>
__global__ void __launch_bounds__(32 * kWarps) wgrad_kernel(const __nv_bfloat16* __restrict__ in,
                                                            const __nv_bfloat16* __restrict__ dout, int N, int H,
                                                            int W, int Cin, int Cout, int chunk,
                                                            float* __restrict__ partial) {
    __shared__ float red[kWarps][16][NT * 8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int tap = blockIdx.y;
    const int ci_tiles = Cin / (NT * 8);
    const int co0 = (blockIdx.z / ci_tiles) * 16, ci0 = (blockIdx.z % ci_tiles) * NT * 8;
    const long long P = (long long)N * H * W;
    const long long p_begin = (long long)blockIdx.x * chunk;
    const long long p_end = p_begin + chunk < P ? p_begin + chunk : P;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    auto shifted = [&](long long p, int ci) -> __nv_bfloat16 {
        if (p >= p_end) return __float2bfloat16_rn(0.0f);
        const int x = (int)(p % W);
        const long long r = p / W;
        const int yv = (int)(r % H);
        const int xs = x + dx, ys = yv + dy;
        if (xs < 0 || xs >= W || ys < 0 || ys >= H) return __float2bfloat16_rn(0.0f);
        return in[(p + (long long)dy * W + dx) * Cin + ci];
    };
    auto dget = [&](long long p, int co) -> __nv_bfloat16 {
        return p < p_end ? dout[p * Cout + co] : __float2bfloat16_rn(0.0f);
    };
    for (long long k0 = p_begin + 16 * warp; k0 < p_end; k0 += 16 * kWarps) {
        // A (16 co x 16 pixels, row-major): rows g, g+8; columns 2t, 2t+1, +8
        uint32_t a[4];
        const long long pk = k0 + 2 * t;
        a[0] = pack2(dget(pk, co0 + g), dget(pk + 1, co0 + g));
        a[1] = pack2(dget(pk, co0 + g + 8), dget(pk + 1, co0 + g + 8));
        a[2] = pack2(dget(pk + 8, co0 + g), dget(pk + 9, co0 + g));
        a[3] = pack2(dget(pk + 8, co0 + g + 8), dget(pk + 9, co0 + g + 8));
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            // B (16 pixels x 8 ci): rows 2t, 2t+1 (+8), column g
            const int ci = ci0 + j * 8 + g;
            uint32_t b[2] = {pack2(shifted(pk, ci), shifted(pk + 1, ci)),
                             pack2(shifted(pk + 8, ci), shifted(pk + 9, ci))};
            mma_bf16(acc[j], a, b);
        }
    }
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        red[warp][g][j * 8 + 2 * t] = acc[j][0];
        red[warp][g][j * 8 + 2 * t + 1] = acc[j][1];
        red[warp][g + 8][j * 8 + 2 * t] = acc[j][2];
        red[warp][g + 8][j * 8 + 2 * t + 1] = acc[j][3];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 16 * NT * 8; e += 32 * kWarps) {
        const int r = e / (NT * 8), c = e % (NT * 8);
        float s = 0.0f;
        for (int q = 0; q < kWarps; ++q) s += red[q][r][c];
        // partial[chunk][co][tap][ci]
        partial[(((size_t)blockIdx.x * Cout + co0 + r) * 9 + tap) * Cin + ci0 + c] = s;
    }
}

// dW = sum of the chunk partials, in a fixed order: thread (column, slice)
// sums four consecutive outputs over the chunks slice, slice + 8, ... and the
// eight slices are then added in slice order.  nw is a multiple of 4.
constexpr int kSlices = 8;

// Blocks past nblocks_w reduce a second array (nb values after the first's
// chunks x nw partials, e.g. the bias partials) into db in the same way.
__global__ void __launch_bounds__(32 * kSlices) wgrad_reduce_kernel(const float* __restrict__ partial, int chunks,
                                                                    size_t nw, float* __restrict__ dw,
                                                                    unsigned nblocks_w = 0, size_t nb = 0,
                                                                    float* __restrict__ db = nullptr) {
    __shared__ float4 red[kSlices][32];
    unsigned blk = blockIdx.x;
    if (db && blk >= nblocks_w) {  // the second array
        partial += (size_t)chunks * nw;
        nw = nb;
        dw = db;
        blk -= nblocks_w;
    }
    const int col = threadIdx.x & 31, slice = threadIdx.x >> 5;
    const size_t i = ((size_t)blk * 32 + col) * 4;
    float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (i < nw) {
#pragma unroll 4
        for (int c = slice; c < chunks; c += kSlices) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(partial + (size_t)c * nw + i));
            s.x += v.x;
            s.y += v.y;
            s.z += v.z;
            s.w += v.w;
        }
    }
    red[slice][col] = s;
    __syncthreads();
    if (slice == 0 && i < nw) {
        float4 t = red[0][col];
        for (int q = 1; q < kSlices; ++q) {
            const float4 v = red[q][col];
            t.x += v.x;
            t.y += v.y;
            t.z += v.z;
            t.w += v.w;
        }
        *reinterpret_cast<float4*>(dw + i) = t;
    }
}

unsigned reduce_blocks(size_t nw) { return (unsigned)((nw / 4 + 31) / 32); }

__global__ void bias_grad_kernel(const __nv_bfloat16* __restrict__ dout, long long P, int Cout, float* __restrict__ db) {
    // one CTA per output channel, fixed-order tree in shared memory
    __shared__ float red[256];
    const int co = blockIdx.x;
    float s = 0.0f;
    for (long long p = threadIdx.x; p < P; p += blockDim.x) s += __bfloat162float(dout[p * Cout + co]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[co] = red[0];
}

// Bias gradient per pixel chunk: thread t sums channel t % Cout over every
// (256 / Cout)-th pixel of the chunk (coalesced rows), the lanes of a channel
// are added in lane order; partial[chunk][co].  Cout divides 256.
__global__ void bias_partial_kernel(const __nv_bfloat16* __restrict__ dout, long long P, int Cout, int chunk,
                                    float* __restrict__ partial) {
    __shared__ float red[256];
    const int lanes = 256 / Cout;
    const int co = threadIdx.x % Cout, lane = threadIdx.x / Cout;
    const long long p0 = (long long)blockIdx.x * chunk;
    const long long p1 = p0 + chunk < P ? p0 + chunk : P;
    float sum = 0.0f;
    for (long long p = p0 + lane; p < p1; p += lanes) sum += __bfloat162float(dout[p * Cout + co]);
    red[threadIdx.x] = sum;
    __syncthreads();
    if (lane == 0) {
        float t = 0.0f;
        for (int l = 0; l < lanes; ++l) t += red[l * Cout + co];
        partial[(size_t)blockIdx.x * Cout + co] = t;
    }
}

// bf16 weights and the data-gradient weights wT[ci][8-tap][co] from the
// float32 master copy w[co][tap][ci]
__global__ void weight_prep_kernel(const float* __restrict__ w, int Cout, int Cin, __nv_bfloat16* __restrict__ wb,
                                   __nv_bfloat16* __restrict__ wt) {
    const size_t n = (size_t)Cout * 9 * Cin;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int ci = (int)(i % Cin);
        const int tap = (int)((i / Cin) % 9);
        const int co = (int)(i / ((size_t)9 * Cin));
        const __nv_bfloat16 v = __float2bfloat16_rn(w[i]);
        wb[i] = v;
        if (wt) wt[((size_t)ci * 9 + (8 - tap)) * Cout + co] = v;
    }
}

// The element-wise kernels below move 8 channels (16 B of bf16, 32 B of
// float32) per thread; every channel count is a multiple of 8.
__device__ __forceinline__ void unpack8(const uint4 v, float f[8]) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        f[2 * k] = __uint_as_float(w[k] << 16);
        f[2 * k + 1] = __uint_as_float(w[k] & 0xFFFF0000u);
    }
}

__device__ __forceinline__ uint4 pack8(const float f[8]) {
    uint32_t w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        w[k] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(f[2 * k])) |
               ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(f[2 * k + 1])) << 16);
    return make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ void load8(const float* p, float f[8]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p)), b = __ldg(reinterpret_cast<const float4*>(p + 4));
    f[0] = a.x, f[1] = a.y, f[2] = a.z, f[3] = a.w, f[4] = b.x, f[5] = b.y, f[6] = b.z, f[7] = b.w;
}

__device__ __forceinline__ void store8(float* p, const float f[8]) {
    reinterpret_cast<float4*>(p)[0] = make_float4(f[0], f[1], f[2], f[3]);
    reinterpret_cast<float4*>(p)[1] = make_float4(f[4], f[5], f[6], f[7]);
}

// 2x2 average pooling (floor sizes), NHWC bf16 -> bf16
__global__ void pool_fwd_kernel(const __nv_bfloat16* __restrict__ in, int N, int H, int W, int C,
                                __nv_bfloat16* __restrict__ out) {
    const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
    const size_t n = (size_t)N * Ho * Wo * C8;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C8) * 8;
        const size_t q = i / C8;
        const int x = (int)(q % Wo), y = (int)((q / Wo) % Ho), b = (int)(q / ((size_t)Wo * Ho));
        const size_t r0 = (((size_t)b * H + 2 * y) * W + 2 * x) * C + c;
        float p00[8], p01[8], p10[8], p11[8], o[8];
        unpack8(__ldg(reinterpret_cast<const uint4*>(in + r0)), p00);
        unpack8(__ldg(reinterpret_cast<const uint4*>(in + r0 + C)), p01);
        unpack8(__ldg(reinterpret_cast<const uint4*>(in + r0 + (size_t)W * C)), p10);
        unpack8(__ldg(reinterpret_cast<const uint4*>(in + r0 + (size_t)W * C + C)), p11);
#pragma unroll
        for (int k = 0; k < 8; ++k) o[k] = 0.25f * ((p00[k] + p01[k]) + (p10[k] + p11[k]));
        *reinterpret_cast<uint4*>(out + q * C + c) = pack8(o);
    }
}

// gradient of the pooling: din (+)= dout / 4 on the pooled pixels, 0 on the dropped edge
__global__ void pool_bwd_kernel(const float* __restrict__ dout, int N, int H, int W, int C, float* __restrict__ din,
                                int accumulate) {
    const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
    const size_t n = (size_t)N * H * W * C8;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C8) * 8;
        const size_t q = i / C8;
        const int x = (int)(q % W), y = (int)((q / W) % H), b = (int)(q / ((size_t)W * H));
        const int xo = x / 2, yo = y / 2;
        float g[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (xo < Wo && yo < Ho) {
            load8(dout + (((size_t)b * Ho + yo) * Wo + xo) * C + c, g);
#pragma unroll
            for (int k = 0; k < 8; ++k) g[k] *= 0.25f;
        }
        float* d = din + q * C + c;
        if (accumulate) {
            float o[8];
            load8(d, o);
#pragma unroll
            for (int k = 0; k < 8; ++k) g[k] += o[k];
        }
        store8(d, g);
    }
}

// out[:, :, :, 0:C1] = nearest 2x upsampling of a (N,Hs,Ws,C1) onto (H,W)
// (source pixel min(y/2, Hs-1), min(x/2, Ws-1)); out[..., C1:C1+C2] = skip
__global__ void upcat_fwd_kernel(const __nv_bfloat16* __restrict__ a, int Hs, int Ws, int C1,
                                 const __nv_bfloat16* __restrict__ skip, int N, int H, int W, int C2,
                                 __nv_bfloat16* __restrict__ out) {
    const int C8 = (C1 + C2) / 8;
    const size_t n = (size_t)N * H * W * C8;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C8) * 8;
        const size_t q = i / C8;
        const int x = (int)(q % W), y = (int)((q / W) % H), b = (int)(q / ((size_t)W * H));
        uint4 v;
        if (c < C1) {
            const int ys = min(y / 2, Hs - 1), xs = min(x / 2, Ws - 1);
            v = __ldg(reinterpret_cast<const uint4*>(a + (((size_t)b * Hs + ys) * Ws + xs) * C1 + c));
        } else {
            v = __ldg(reinterpret_cast<const uint4*>(skip + q * C2 + (c - C1)));
        }
        reinterpret_cast<uint4*>(out)[i] = v;
    }
}

// gradient of upcat: da (+)= sum of the fine pixels that copy each coarse one;
// dskip += dout[..., C1:]
__global__ void upcat_bwd_a_kernel(const float* __restrict__ dout, int N, int H, int W, int C1, int C2, int Hs,
                                   int Ws, float* __restrict__ da, int accumulate) {
    const int C = C1 + C2, C8 = C1 / 8;
    const size_t n = (size_t)N * Hs * Ws * C8;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C8) * 8;
        const size_t q = i / C8;
        const int xs = (int)(q % Ws), ys = (int)((q / Ws) % Hs), b = (int)(q / ((size_t)Ws * Hs));
        const int ya = 2 * ys, yb = (ys == Hs - 1) ? H : min(2 * ys + 2, H);
        const int xa = 2 * xs, xb = (xs == Ws - 1) ? W : min(2 * xs + 2, W);
        float s[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        for (int y = ya; y < yb; ++y)
            for (int x = xa; x < xb; ++x) {
                float g[8];
                load8(dout + (((size_t)b * H + y) * W + x) * C + c, g);
#pragma unroll
                for (int k = 0; k < 8; ++k) s[k] += g[k];
            }
        float* d = da + q * C1 + c;
        if (accumulate) {
            float o[8];
            load8(d, o);
#pragma unroll
            for (int k = 0; k < 8; ++k) s[k] = o[k] + s[k];
        }
        store8(d, s);
    }
}

__global__ void upcat_bwd_skip_kernel(const float* __restrict__ dout, size_t npix, int C1, int C2,
                                      float* __restrict__ dskip, int accumulate) {
    const int C8 = C2 / 8;
    const size_t n = npix * C8;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i / C8;
        const int c = (int)(i % C8) * 8;
        float g[8];
        load8(dout + p * (C1 + C2) + C1 + c, g);
        float* d = dskip + p * C2 + c;
        if (accumulate) {
            float o[8];
            load8(d, o);
#pragma unroll
            for (int k = 0; k < 8; ++k) g[k] = o[k] + g[k];
        }
        store8(d, g);
    }
}

// dpre = da * (a > 0) as bf16 (the ReLU gradient, a the stored activation); n a multiple of 8
__global__ void relu_bwd_kernel(const float* __restrict__ da, const __nv_bfloat16* __restrict__ a, size_t n,
                                __nv_bfloat16* __restrict__ dpre) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n / 8; i += (size_t)gridDim.x * blockDim.x) {
        float g[8], v[8];
        load8(da + 8 * i, g);
        unpack8(__ldg(reinterpret_cast<const uint4*>(a) + i), v);
#pragma unroll
        for (int k = 0; k < 8; ++k) g[k] = v[k] > 0.0f ? g[k] : 0.0f;
        reinterpret_cast<uint4*>(dpre)[i] = pack8(g);
    }
}

// Mean-squared error of channel 0 of out32 ([P, C]) against target [P] on the
// masked pixels: per-CTA FP64 partials; dout (bf16 [P, C]) gets
// 2 (out - target) * scale on channel 0 and zero elsewhere.
__global__ void mse_kernel(const float* __restrict__ out32, int C, const float* __restrict__ target,
                           const float* __restrict__ mask, long long P, float scale, __nv_bfloat16* __restrict__ dout,
                           double* __restrict__ partial) {
    __shared__ double red[256];
    double s = 0.0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        const float m = mask ? mask[p] : 1.0f;
        const float d = (out32[p * C] - target[p]) * m;
        s += (double)d * (double)d;
        uint4* o = reinterpret_cast<uint4*>(dout + p * C);  // C a multiple of 8
        o[0] = make_uint4((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(2.0f * d * scale)), 0u, 0u, 0u);
        for (int c = 1; c < C / 8; ++c) o[c] = make_uint4(0u, 0u, 0u, 0u);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void sum_partials_kernel(const double* __restrict__ partial, int n, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += partial[i];
        *out = s;
    }
}

// Adam (Kingma & Ba 2015) on float32 master weights
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// Network input from three nz x nx float32 grids (z fastest, i.e. W = nz runs
// fastest) into NHWC bf16 with C = 16, image row = model column x, image
// column = depth z:
//   ch0 = q / max|q|, q = g / (il + 1e-3 max il)  (illumination-balanced gradient)
//   ch1 = 1 + log10(il / max il + 1e-6) / 6       (illumination, 0..1)
//   ch2 = (v - v0) * vs                            (velocity)
// channels 3..15 zero.  Pass 1 finds max il, pass 2 max |q| (bits[0], bits[1]).
__device__ __forceinline__ float balanced(float g, float il, float ilmax) { return g / (il + 1e-3f * ilmax); }

__global__ void pack_max_il_kernel(const float* __restrict__ il, size_t n, unsigned* bits) {
    float m = 0.0f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(il[p]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(bits, __float_as_uint(m));
}

__global__ void pack_max_q_kernel(const float* __restrict__ g, const float* __restrict__ il, size_t n,
                                  unsigned* bits) {
    const float ilmax = __uint_as_float(bits[0]);
    float m = 0.0f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(balanced(g[p], fabsf(il[p]), ilmax)));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(bits + 1, __float_as_uint(m));
}

__global__ void pack_inputs_kernel(const float* __restrict__ g, const float* __restrict__ il,
                                   const float* __restrict__ v, size_t n, float v0, float vs,
                                   const unsigned* __restrict__ bits, __nv_bfloat16* __restrict__ out) {
    const float ilmax = fmaxf(__uint_as_float(bits[0]), 1e-30f);
    const float qs = 1.0f / fmaxf(__uint_as_float(bits[1]), 1e-30f);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const float a = fabsf(il[p]);
        __nv_bfloat16* o = out + p * 16;
        o[0] = __float2bfloat16_rn(balanced(g[p], a, ilmax) * qs);
        o[1] = __float2bfloat16_rn(1.0f + log10f(a / ilmax + 1e-6f) / 6.0f);
        o[2] = __float2bfloat16_rn((v[p] - v0) * vs);
        for (int c = 3; c < 16; ++c) o[c] = __float2bfloat16_rn(0.0f);
    }
}

__global__ void unpack_kernel(const float* __restrict__ out32, int C, long long P, float* __restrict__ dst) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
        dst[p] = out32[p * C];
}

unsigned grid_n(size_t n) {
    size_t b = (n + 255) / 256;
    if (b == 0) b = 1;
    return (unsigned)(b < 148 * 32 ? b : 148 * 32);
}

}  // namespace

int nn_conv3x3_mma(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout,
                   int relu, void* out, float* out32, cudaStream_t st) {
    if (Cin % 16 || Cout % 16 || N < 1 || H < 1 || W < 1) return -1;
    const int runs = (W + 15) / 16;
    const int xb = (runs + kWarps - 1) / kWarps;
    const auto* i16 = static_cast<const __nv_bfloat16*>(in);
    const auto* w16 = static_cast<const __nv_bfloat16*>(w);
    auto* o16 = static_cast<__nv_bfloat16*>(out);
    if (Cout % 32 == 0) {
        dim3 grid(xb * N, H, Cout / 32);
        conv3x3_kernel<4><<<grid, 32 * kWarps, 0, st>>>(i16, N, H, W, Cin, w16, bias, Cout, relu, o16, out32);
    } else {
        dim3 grid(xb * N, H, Cout / 16);
        conv3x3_kernel<2><<<grid, 32 * kWarps, 0, st>>>(i16, N, H, W, Cin, w16, bias, Cout, relu, o16, out32);
    }
    return 0;
}

int nn_wgrad_chunks(long long P) {
    long long c = (P + 1023) / 1024;  // ~1024 pixels per chunk
    return (int)(c < 512 ? (c < 1 ? 1 : c) : 512);
}

int nn_conv3x3_wgrad(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, float* partial,
                     float* dw, float* db, cudaStream_t st, bool tensor_memory) {
    if (Cin % 16 || Cout % 16) return -1;
    const long long P = (long long)N * H * W;
    const int chunks = nn_wgrad_chunks(P);
    const int chunk = (int)(((P + chunks - 1) / chunks + 15) / 16 * 16);
    const auto* i16 = static_cast<const __nv_bfloat16*>(in);
    const auto* d16 = static_cast<const __nv_bfloat16*>(dout);
    const size_t nw = (size_t)Cout * 9 * Cin;
    // the tcgen05 kernel takes up to 128 output channels and sums the bias
    // gradient too; wider layers, and callers asking for the mma.sync path,
    // use the warp-level kernel
    if (tensor_memory && Cout <= 128) {
        const int tc_chunks = nn_wgrad_tma(in, dout, N, H, W, Cin, Cout, partial, db != nullptr, st);
        if (tc_chunks == -2) return -2;
        if (tc_chunks > 0) {
            // the weight partials, then (db) the bias partials stored after them, in one launch
            const unsigned bw = reduce_blocks(nw), bb = db ? reduce_blocks((size_t)Cout) : 0u;
            wgrad_reduce_kernel<<<bw + bb, 32 * kSlices, 0, st>>>(partial, tc_chunks, nw, dw, bw, (size_t)Cout, db);
            return 0;
        }
    }
    if (Cin % 32 == 0) {
        dim3 grid(chunks, 9, (Cout / 16) * (Cin / 32));
        wgrad_kernel<4><<<grid, 32 * kWarps, 0, st>>>(i16, d16, N, H, W, Cin, Cout, chunk, partial);
    } else {
        dim3 grid(chunks, 9, (Cout / 16) * (Cin / 16));
        wgrad_kernel<2><<<grid, 32 * kWarps, 0, st>>>(i16, d16, N, H, W, Cin, Cout, chunk, partial);
    }
    wgrad_reduce_kernel<<<reduce_blocks(nw), 32 * kSlices, 0, st>>>(partial, chunks, nw, dw);
    if (db) {
        if (256 % Cout == 0) {  // the chunk partials are consumed: reuse the scratch
            bias_partial_kernel<<<chunks, 256, 0, st>>>(d16, P, Cout, chunk, partial);
            wgrad_reduce_kernel<<<reduce_blocks((size_t)Cout), 32 * kSlices, 0, st>>>(partial, chunks, (size_t)Cout, db);
        } else {
            bias_grad_kernel<<<Cout, 256, 0, st>>>(d16, P, Cout, db);
        }
    }
    return 0;
}

void nn_weight_prep(const float* w, int Cout, int Cin, void* wb, void* wt, cudaStream_t st) {
    const size_t n = (size_t)Cout * 9 * Cin;
    weight_prep_kernel<<<grid_n(n), 256, 0, st>>>(w, Cout, Cin, static_cast<__nv_bfloat16*>(wb),
                                                   static_cast<__nv_bfloat16*>(wt));
}

void nn_pool_fwd(const void* in, int N, int H, int W, int C, void* out, cudaStream_t st) {
    pool_fwd_kernel<<<grid_n((size_t)N * (H / 2) * (W / 2) * C / 8), 256, 0, st>>>(
        static_cast<const __nv_bfloat16*>(in), N, H, W, C, static_cast<__nv_bfloat16*>(out));
}

void nn_pool_bwd(const float* dout, int N, int H, int W, int C, float* din, int accumulate, cudaStream_t st) {
    pool_bwd_kernel<<<grid_n((size_t)N * H * W * C / 8), 256, 0, st>>>(dout, N, H, W, C, din, accumulate);
}

void nn_upcat_fwd(const void* a, int Hs, int Ws, int C1, const void* skip, int N, int H, int W, int C2, void* out,
                  cudaStream_t st) {
    upcat_fwd_kernel<<<grid_n((size_t)N * H * W * (C1 + C2) / 8), 256, 0, st>>>(
        static_cast<const __nv_bfloat16*>(a), Hs, Ws, C1, static_cast<const __nv_bfloat16*>(skip), N, H, W, C2,
        static_cast<__nv_bfloat16*>(out));
}

void nn_upcat_bwd(const float* dout, int N, int H, int W, int C1, int C2, int Hs, int Ws, float* da, int acc_a,
                  float* dskip, int acc_skip, cudaStream_t st) {
    upcat_bwd_a_kernel<<<grid_n((size_t)N * Hs * Ws * C1 / 8), 256, 0, st>>>(dout, N, H, W, C1, C2, Hs, Ws, da, acc_a);
    upcat_bwd_skip_kernel<<<grid_n((size_t)N * H * W * C2 / 8), 256, 0, st>>>(dout, (size_t)N * H * W, C1, C2, dskip,
                                                                         acc_skip);
}

void nn_relu_bwd(const float* da, const void* a, size_t n, void* dpre, cudaStream_t st) {
    relu_bwd_kernel<<<grid_n(n / 8), 256, 0, st>>>(da, static_cast<const __nv_bfloat16*>(a), n,
                                               static_cast<__nv_bfloat16*>(dpre));
}

void nn_mse(const float* out32, int C, const float* target, const float* mask, long long P, float scale, void* dout,
            double* partial, double* loss, cudaStream_t st) {
    const int blocks = 256;
    mse_kernel<<<blocks, 256, 0, st>>>(out32, C, target, mask, P, scale, static_cast<__nv_bfloat16*>(dout), partial);
    sum_partials_kernel<<<1, 32, 0, st>>>(partial, blocks, loss);
}

void nn_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps, int step,
             cudaStream_t st) {
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    adam_kernel<<<grid_n(n), 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2);
}

void nn_pack_inputs(const float* g, const float* il, const float* v, int nz, int nx, float v0, float vs,
                    unsigned* bits, void* out, cudaStream_t st) {
    const size_t n = (size_t)nz * nx;
    cudaMemsetAsync(bits, 0, 2 * sizeof(unsigned), st);
    pack_max_il_kernel<<<grid_n(n), 256, 0, st>>>(il, n, bits);
    pack_max_q_kernel<<<grid_n(n), 256, 0, st>>>(g, il, n, bits);
    pack_inputs_kernel<<<grid_n(n), 256, 0, st>>>(g, il, v, n, v0, vs, bits, static_cast<__nv_bfloat16*>(out));
}

void nn_unpack_channel(const float* out32, int C, long long P, float* dst, cudaStream_t st) {
    unpack_kernel<<<grid_n((size_t)P), 256, 0, st>>>(out32, C, P, dst);
}

}  // namespace fwi
