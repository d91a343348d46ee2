// k_nn_tc.cu — the U-Net's 3x3 convolutions on the 5th-generation tensor
// cores (tcgen05, accumulators in tensor memory).
//
// Implicit GEMM: D[p, co] = sum_{tap, ci} A_tap[p, ci] B_tap[co, ci], with
// A_tap[p, ci] = in[p shifted by the tap, ci] (zero outside the image) and
// B_tap[co, ci] = w[co, tap, ci].  A CTA owns M = 128 consecutive pixels of
// the flattened N x H x W image (rows of the tile may cross image rows) and
// all Cout output channels (N = Cout <= 256, a multiple of 16):
//
//   * per tap, the 128 threads stage A_tap (128 x Cin) and B_tap (Cout x Cin)
//     in shared memory in the canonical K-major layout without swizzle
//     (8-row x 16-byte core matrices; K-adjacent core matrices 128 B apart,
//     8-row groups Cin/8 x 128 B apart) with 16-byte cp.async copies (zero
//     fill outside the image), all of a tap's copies in flight at once, two
//     stages so the copies of tap t+1 overlap the MMAs of tap t;
//   * one thread issues the tap's Cin/16 `tcgen05.mma.cta_group::1.kind::f16`
//     (BF16 x BF16 -> FP32, M = 128, N = Cout) into a TMEM accumulator and
//     commits them to the stage's mbarrier;
//   * after the last tap each warp reads its 32 TMEM lanes (pixels) with
//     `tcgen05.ld.32x32b`, adds the bias, applies the ReLU and stores bf16 /
//     float32 NHWC rows.
// Every mbarrier wait is bounded; a wait that gives up raises g_tc_err
// (fwi_nn_check) and the CTA still waits (bounded) before freeing its TMEM.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"
#include "tma.cuh"

namespace fwi {

namespace {

constexpr int kTcM = 128;        // pixels per CTA tile = TMEM lanes
constexpr int kTcThreads = 128;  // 4 warps; warp w reads TMEM lanes 32w..32w+31

__device__ int g_tc_err;

__device__ __forceinline__ uint32_t saddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: canonical K-major layout, no swizzle,
// descriptor version 1 (sm_100), base offset 0.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N and M as given.
__device__ __forceinline__ uint32_t umma_idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    const uint32_t mask[4] = {0u, 0u, 0u, 0u};
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(mask[0]), "r"(mask[1]), "r"(mask[2]),
          "r"(mask[3]));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t addr, uint32_t r[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16-byte asynchronous copy global -> shared memory (L2 only); src_bytes 0
// writes zeros (the source address must still be a valid one).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
// Wait for every cp.async of the thread, then make the copies visible to the
// tensor cores' (async proxy) reads.
__device__ __forceinline__ void cp_async_wait_all_async_proxy() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

__global__ void __launch_bounds__(kTcThreads) conv3x3_tc_kernel(const __nv_bfloat16* __restrict__ in, int N, int H,
                                                                int W, int Cin, const __nv_bfloat16* __restrict__ w,
                                                                const float* __restrict__ bias, int Cout, int ncols,
                                                                uint32_t stage_bytes, int relu,
                                                                __nv_bfloat16* __restrict__ out,
                                                                float* __restrict__ out32) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long P = (long long)N * H * W;
    const long long p = (long long)blockIdx.x * kTcM + tid;  // this thread's pixel (A row, TMEM lane)
    const int kc = Cin / 8;
    const uint32_t a_bytes = (uint32_t)kTcM * Cin * 2;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_slot)),
                     "r"(ncols)
                     : "memory");
        tc_fence_before();
    }
    if (tid == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    const bool valid = p < P;
    int n = 0, y = 0, x = 0;
    if (valid) {
        x = (int)(p % W);
        const long long r = p / W;
        y = (int)(r % H);
        n = (int)(r / H);
    }
    const uint32_t idesc = umma_idesc(kTcM, Cout);
    bool ok = true;
    for (int tap = 0; tap < 9; ++tap) {
        const int s = tap & 1;
        unsigned char* A = smem + (size_t)s * stage_bytes;
        unsigned char* B = A + a_bytes;
        // the stage's previous MMAs (tap - 2) must be done before it is rewritten
        if (tap >= 2 && !tma::mbar_wait(&bar[s], (uint32_t)(((tap - 2) >> 1) & 1))) ok = false;
        const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
        const bool in_ok = valid && yy >= 0 && yy < H && xx >= 0 && xx < W;
        const uint4* src = reinterpret_cast<const uint4*>(in + (((long long)n * H + (in_ok ? yy : 0)) * W +
                                                                (in_ok ? xx : 0)) * Cin);
        unsigned char* arow = A + (size_t)(tid >> 3) * kc * 128 + (tid & 7) * 16;
        const uint32_t a_src = in_ok ? 16u : 0u;
        for (int j = 0; j < kc; ++j) cp_async16(arow + (size_t)j * 128, src + j, a_src);
        for (int e = tid; e < Cout * kc; e += kTcThreads) {
            const int co = e / kc, j = e - co * kc;
            cp_async16(B + ((size_t)(co >> 3) * kc + j) * 128 + (co & 7) * 16,
                       reinterpret_cast<const uint4*>(w + ((long long)co * 9 + tap) * Cin) + j, 16u);
        }
        cp_async_wait_all_async_proxy();  // the tensor cores read these copies through the async proxy
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sa = saddr(A), sb = saddr(B);
            for (int k = 0; k < Cin / 16; ++k)
                umma_bf16(tmem, umma_desc(sa + 256u * k, 128u, (uint32_t)kc * 128u),
                          umma_desc(sb + 256u * k, 128u, (uint32_t)kc * 128u), idesc, (tap | k) != 0 ? 1u : 0u);
            umma_commit(&bar[s]);
        }
    }
    // tap 8 (stage 0, its 5th use) commits after every earlier MMA; the last
    // arrival on stage 1 (tap 7) is collected too, so none lands after exit
    if (!tma::mbar_wait(&bar[0], 0u)) ok = false;
    if (!tma::mbar_wait(&bar[1], 1u)) ok = false;
    tc_fence_after();
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < Cout; c0 += 8) {
        uint32_t r[8];
        tmem_ld8(lane_addr + (uint32_t)c0, r);
        if (!valid) continue;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float t = __uint_as_float(r[j]);
            if (bias) t += __ldg(bias + c0 + j);
            if (relu) t = fmaxf(t, 0.0f);
            v[j] = t;
        }
        if (out)
            *reinterpret_cast<uint4*>(out + p * Cout + c0) =
                make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                           pack_bf16x2(v[6], v[7]));
        if (out32) {
            float4* o = reinterpret_cast<float4*>(out32 + p * Cout + c0);
            o[0] = make_float4(v[0], v[1], v[2], v[3]);
            o[1] = make_float4(v[4], v[5], v[6], v[7]);
        }
    }
    if (!ok) atomicExch(&g_tc_err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}

// Weight gradient of the same convolution on the tensor cores:
//   dW[co, tap, ci] = sum_p dout[p, co] in[p + tap, ci]
// a GEMM with M = co (padded to 128), N = ci, K = pixels.  Both operands are
// MN-major in memory (NHWC: channels contiguous for a pixel), so they are
// staged in the canonical MN-major layout without swizzle: core matrices of
// 8 pixels (K rows) x 16 bytes (8 channels); K-adjacent core matrices 128 B
// apart, channel-adjacent ones 1024 B apart (8 K groups = 64 pixels per
// stage).  CTA (chunk, tap) accumulates its pixel chunk in TMEM and writes
// the float32 partial[chunk][co][tap][ci]; chunks are summed in a fixed order
// afterwards (wgrad_reduce_kernel in k_nn.cu).
constexpr int kWgK = 64;  // pixels per stage

__global__ void __launch_bounds__(kTcThreads) wgrad_tc_kernel(const __nv_bfloat16* __restrict__ in,
                                                              const __nv_bfloat16* __restrict__ dout, int N, int H,
                                                              int W, int Cin, int Cout, int chunk, int ncols,
                                                              uint32_t stage_bytes, float* __restrict__ partial) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tap = blockIdx.y;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    const long long P = (long long)N * H * W;
    const long long p_begin = (long long)blockIdx.x * chunk;
    const long long p_end = p_begin + chunk < P ? p_begin + chunk : P;
    const uint32_t a_bytes = 16u * 8u * 128u;  // 128 co x 64 pixels
    const int nci = Cin / 8;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_slot)),
                     "r"(ncols)
                     : "memory");
        tc_fence_before();
    }
    if (tid == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    // M = 128, N = Cin, both operands MN-major (bits 15 and 16)
    const uint32_t idesc = umma_idesc(128, Cin) | (1u << 15) | (1u << 16);
    const int nstage = p_end > p_begin ? (int)((p_end - p_begin + kWgK - 1) / kWgK) : 0;
    // the output-channel groups past Cout (M is padded to 128) hold zeros in
    // both stages for the whole launch: cleared once here, never copied
    const int mgroups = (Cout + 7) / 8;
    for (int s = 0; s < 2; ++s) {
        uint4* pad = reinterpret_cast<uint4*>(smem + (size_t)s * stage_bytes + (size_t)mgroups * 8 * 128);
        for (int i = tid; i < (16 - mgroups) * 8 * 8; i += kTcThreads) pad[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    bool ok = true;
    for (int st = 0; st < nstage; ++st) {
        const int s = st & 1;
        unsigned char* A = smem + (size_t)s * stage_bytes;
        unsigned char* B = A + a_bytes;
        if (st >= 2 && !tma::mbar_wait(&bar[s], (uint32_t)(((st - 2) >> 1) & 1))) ok = false;
        const long long q0 = p_begin + (long long)st * kWgK;
        // A: dout rows (pixels) x co, the Cout / 8 real co groups x 64 pixels
        // (zeros past the chunk; the copy's source is then pixel p_begin, channel 0)
        for (int e = tid; e < mgroups * kWgK; e += kTcThreads) {
            const int mi = e / kWgK, r = e - mi * kWgK;  // co group, pixel in stage
            const long long q = q0 + r;
            const bool ok_a = q < p_end;
            cp_async16(A + ((size_t)mi * 8 + (r >> 3)) * 128 + (r & 7) * 16,
                       reinterpret_cast<const uint4*>(dout + (ok_a ? q * Cout + mi * 8 : p_begin * Cout)),
                       ok_a ? 16u : 0u);
        }
        // B: shifted input rows (pixels) x ci (zeros outside the image)
        for (int e = tid; e < nci * kWgK; e += kTcThreads) {
            const int ni = e / kWgK, r = e - ni * kWgK;
            const long long q = q0 + r;
            bool ok_b = false;
            if (q < p_end) {
                const int x = (int)(q % W);
                const int y = (int)((q / W) % H);
                ok_b = x + dx >= 0 && x + dx < W && y + dy >= 0 && y + dy < H;
            }
            cp_async16(B + ((size_t)ni * 8 + (r >> 3)) * 128 + (r & 7) * 16,
                       reinterpret_cast<const uint4*>(in + (ok_b ? (q + (long long)dy * W + dx) * Cin + ni * 8 : 0)),
                       ok_b ? 16u : 0u);
        }
        cp_async_wait_all_async_proxy();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sa = saddr(A), sb = saddr(B);
            for (int k = 0; k < kWgK / 16; ++k)
                umma_bf16(tmem, umma_desc(sa + 256u * k, 128u, 1024u), umma_desc(sb + 256u * k, 128u, 1024u), idesc,
                          (st | k) != 0 ? 1u : 0u);
            umma_commit(&bar[s]);
        }
    }
    // collect the last use of each stage
    for (int s = 0; s < 2; ++s) {
        const int last = nstage - 1 - ((nstage - 1 - s) & 1);  // last stage index with parity s
        if (last >= 0 && last % 2 == s && !tma::mbar_wait(&bar[s], (uint32_t)((last >> 1) & 1))) ok = false;
    }
    tc_fence_after();
    const int co = tid;  // TMEM lane = output channel
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < Cin; c0 += 8) {
        uint32_t r[8];
        tmem_ld8(lane_addr + (uint32_t)c0, r);
        if (co >= Cout) continue;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = nstage > 0 ? __uint_as_float(r[j]) : 0.0f;
        float4* o = reinterpret_cast<float4*>(partial + (((size_t)blockIdx.x * Cout + co) * 9 + tap) * Cin + c0);
        o[0] = make_float4(v[0], v[1], v[2], v[3]);
        o[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
    if (!ok) atomicExch(&g_tc_err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}

}  // namespace

int nn_wgrad_tc(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, int chunks, int chunk,
                float* partial, cudaStream_t st) {
    if (Cin % 16 || Cin > 256 || Cout % 16 || Cout > 128 || chunks < 1 || chunk % 16) return -1;
    int ncols = 32;
    while (ncols < Cin) ncols *= 2;
    const uint32_t stage = 16u * 8u * 128u + (uint32_t)Cin * 128u;
    size_t smem = 2 * (size_t)stage;
    const size_t tmem_share = (size_t)ncols * 460;
    if (smem < tmem_share) smem = tmem_share;
    static size_t configured = 0;
    if (smem > configured) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, wgrad_tc_kernel) != cudaSuccess) return -2;
        if (smem + fa.sharedSizeBytes > 227 * 1024) return -1;
        if (cudaFuncSetAttribute(wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return -2;
        configured = smem;
    }
    wgrad_tc_kernel<<<dim3(chunks, 9), kTcThreads, smem, st>>>(static_cast<const __nv_bfloat16*>(in),
                                                               static_cast<const __nv_bfloat16*>(dout), N, H, W, Cin,
                                                               Cout, chunk, ncols, stage, partial);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int nn_conv3x3_tc(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout, int relu,
                  void* out, float* out32, cudaStream_t st) {
    if (Cin % 16 || Cin > 256 || Cout % 16 || Cout > 256 || N < 1 || H < 1 || W < 1) return -1;
    int ncols = 32;
    while (ncols < Cout) ncols *= 2;
    const uint32_t stage = ((uint32_t)(kTcM * Cin + Cout * Cin) * 2u + 1023u) / 1024u * 1024u;
    // at most 512 TMEM columns of resident CTAs per SM: ask for enough shared
    // memory that no more CTAs than that fit
    size_t smem = 2 * (size_t)stage;
    const size_t tmem_share = (size_t)ncols * 460;
    if (smem < tmem_share) smem = tmem_share;
    // dynamic shared memory above the default needs the attribute (the
    // static 1 KB of barriers and alignment comes on top of it)
    static size_t configured = 0;
    if (smem > configured) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, conv3x3_tc_kernel) != cudaSuccess) return -2;
        if (smem + fa.sharedSizeBytes > 227 * 1024) return -1;  // two stages do not fit: unsupported size
        if (cudaFuncSetAttribute(conv3x3_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return -2;
        configured = smem;
    }
    const long long P = (long long)N * H * W;
    const unsigned grid = (unsigned)((P + kTcM - 1) / kTcM);
    conv3x3_tc_kernel<<<grid, kTcThreads, smem, st>>>(
        static_cast<const __nv_bfloat16*>(in), N, H, W, Cin, static_cast<const __nv_bfloat16*>(w), bias, Cout, ncols,
        stage, relu, static_cast<__nv_bfloat16*>(out), out32);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int nn_tc_error(bool reset) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_tc_err, sizeof(int)) != cudaSuccess) return -1;
    if (reset && v) {
        const int z = 0;
        cudaMemcpyToSymbol(g_tc_err, &z, sizeof(int));
    }
    return v;
}

}  // namespace fwi
