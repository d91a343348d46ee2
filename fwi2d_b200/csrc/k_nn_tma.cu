// k_nn_tma.cu — the U-Net's 3x3 convolutions and weight gradients on the
// 5th-generation tensor cores, operands brought in by TMA, warp-specialised:
// warp 0 (one lane) issues the TMA loads into a ring of mbarrier stages,
// warp 1 (one lane) the `tcgen05.mma.kind::f16` (BF16 x BF16 -> FP32 in
// tensor memory) and the commits, warps 2-5 read the accumulators back with
// `tcgen05.ld.32x32b` (each its 32-lane quarter).  CTAs are persistent, one
// per SM.  Every fixed cost here is per instruction of one thread (about
// 60 ns a TMA load, 35-50 ns an MMA on this part, plus the thread's own
// integer work: descriptors are built once and offset by constants), so the
// kernels are shaped to issue few, wide operations per pixel.
//
// Convolution D[p, co] = sum_{tap, ci} in[p + tap, ci] w[co, tap, ci], two kernels:
//   * conv3x3_halo_kernel (the weights fit in shared memory next to the
//     ring): a tile is 8 x 16 pixels; its input plus a one-pixel border is
//     loaded once, one box per 8-channel plane, in the no-swizzle canonical
//     layout, and the nine taps read it through shifted descriptors; the
//     weights stay resident for the CTA's life;
//   * conv3x3_tma_kernel (large weights): a tile is a bw x bh box of 128
//     pixels; per (tap, channel block of 64 / 32 / 16) one swizzled 4-D box of
//     the shifted pixels (zero fill gives the padding) and one of the weights,
//     or, with 64-channel blocks, one 5-D box of several blocks and one 4-D
//     box of their weights per stage.
//   Both keep two TMEM accumulators (M = 128 lanes x Cout columns) so the
//   epilogue of a tile (bias, ReLU, NHWC store) overlaps the next tile's MMAs.
//
// Weight gradient dW[co, tap, ci] = sum_p dout[p, co] in[p + tap, ci]:
//   M = co (128 TMEM lanes; rows past Cout are ignored), K = pixels in boxes of
//   128.  CTA (chunk, tap group) streams the boxes of its pixel chunk: per
//   stage one output-gradient box (MN-major A) and one shifted input box per
//   tap of its group (MN-major B).  The taps' input boxes sit back to back, so
//   up to 256 / Cin taps form one MMA (N = taps x Cin) whose accumulator
//   columns come out in [tap][ci] order; the bias gradient rides along as one
//   more MMA against a block of ones.  The partials [chunk][co][tap][ci] and
//   [chunk][co] are summed over chunks in a fixed order afterwards.
//
// Every wait is bounded (tma::kSpinLimit polls); a wait that gives up raises
// g_nn_tma_err (fwi_nn_check), the roles stop issuing, the producer collects
// its copies in flight and the MMA thread its last commit before the TMEM is
// freed.  No load uses .multicast::cluster.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"
#include "tma.cuh"

namespace fwi {

namespace {

constexpr int kThreads = 192;     // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int kMaxStages = 32;
constexpr int kConvM = 128;       // pixels per convolution tile = TMEM lanes
constexpr int kWgK = 128;         // pixels per weight-gradient stage
constexpr uint32_t kOnesBytes = 1024;

__device__ int g_nn_tma_err;

// ----------------------------------------------------------------- tcgen05
__device__ __forceinline__ uint32_t saddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// sm_100 shared-memory matrix descriptor: start, leading / stride byte
// offsets, version 1, base offset 0, layout type (0 none, 2 128B, 4 64B,
// 6 32B swizzle) in bits 61-63.
__device__ __forceinline__ uint64_t mdesc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}

__device__ __forceinline__ uint32_t layout_of(int sw) { return sw == 128 ? 2u : sw == 64 ? 4u : 6u; }

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// A / B MN-major when a_mn / b_mn, N and M as given.
__device__ __forceinline__ uint32_t idesc(int m, int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn ? 1u << 15 : 0u) | (b_mn ? 1u << 16 : 0u) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t id, bool acc) {
    const uint32_t z = 0u;  // no output lane disabled
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(id), "r"(acc ? 1u : 0u), "r"(z));
}

__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t addr, uint32_t r[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, int ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t addr, int ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(addr), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

__device__ __forceinline__ unsigned char* align1024(unsigned char* p) {
    return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~(uintptr_t)1023);
}

// ------------------------------------------------------------ convolution
struct ConvArgs {
    int H, W, Cout;
    int bw, tiles_x, tiles_y, ntiles;
    int cb, nkb, sw;  // channels per block, blocks per tap, row bytes (= 2 cb)
    int bps;          // channel blocks per stage (> 1: one 5-D input box and one 4-D weight box per stage)
    int stages;
    uint32_t stage_bytes, a_bytes, tx_bytes;  // a_bytes: the stage's input boxes
    int ncols;  // TMEM columns allocated (>= 2 Cout)
    const float* bias;
    int relu;
    __nv_bfloat16* out;
    float* out32;
};

__device__ __forceinline__ void conv_tile_origin(const ConvArgs& a, int t, int& n, int& x0, int& y0) {
    const int tx = t % a.tiles_x;
    const int r = t / a.tiles_x;
    x0 = tx * a.bw;
    y0 = (r % a.tiles_y) * (kConvM / a.bw);
    n = r / a.tiles_y;
}

__global__ void __launch_bounds__(kThreads, 1)
    conv3x3_tma_kernel(const __grid_constant__ CUtensorMap m_in, const __grid_constant__ CUtensorMap m_w,
                       const ConvArgs a) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = align1024(smem_raw);
    __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], tfull[2], tempty[2], fin;
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 1) {
        tmem_alloc(&tmem_slot, a.ncols);
        fence_before();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < a.stages; ++s) {
            tma::mbar_init(&full[s], 1);
            tma::mbar_init(&empty[s], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tma::mbar_init(&tfull[i], 1);
            tma::mbar_init(&tempty[i], 4);
        }
        tma::mbar_init(&fin, 1);
        tma::fence_barrier_init();
        tma::prefetch_map(&m_in);
        tma::prefetch_map(&m_w);
    }
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    const int spt = a.nkb / a.bps;  // stages per tap
    const int nk = 9 * spt;         // stages per tile
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t it = 0;
            for (int t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x) {
                int n, x0, y0;
                conv_tile_origin(a, t, n, x0, y0);
                for (int kk = 0; kk < nk; ++kk, ++it) {
                    const int tap = kk / spt, kb = (kk - tap * spt) * a.bps;  // first channel block of the stage
                    const int s = (int)(it % (uint32_t)a.stages);
                    const uint32_t use = it / (uint32_t)a.stages;
                    if (!tma::mbar_wait(&empty[s], (use & 1u) ^ 1u)) {
                        ok = false;
                        break;
                    }
                    unsigned char* A = smem + (size_t)s * a.stage_bytes;
                    tma::mbar_arrive_expect_tx(&full[s], a.tx_bytes);
                    if (a.bps == 1) {
                        tma::load_4d(A, &m_in, kb * a.cb, x0 + tap % 3 - 1, y0 + tap / 3 - 1, n, &full[s]);
                        tma::load_3d(A + a.a_bytes, &m_w, kb * a.cb, tap, 0, &full[s]);
                    } else {
                        // (channel, x, y, image, block) and (channel, co, tap, block): bps blocks back to back
                        tma::load_5d(A, &m_in, 0, x0 + tap % 3 - 1, y0 + tap / 3 - 1, n, kb, &full[s]);
                        tma::load_4d(A + a.a_bytes, &m_w, 0, 0, tap, kb, &full[s]);
                    }
                }
            }
            // the last fill of every stage has landed before the CTA can exit
            for (int s = 0; s < a.stages; ++s)
                if ((uint32_t)s < it && !tma::mbar_wait(&full[s], ((it - 1 - s) / (uint32_t)a.stages) & 1u)) ok = false;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t id = idesc(kConvM, a.Cout, false, false);
            const uint32_t lay = layout_of(a.sw), sbo = 8u * (uint32_t)a.sw;
            // the A and B descriptors of stage 0, block 0; others are constant offsets
            const uint64_t d0 = mdesc(saddr(smem), 16u, sbo, lay);
            const uint64_t blk_a = ((uint64_t)kConvM * a.sw) >> 4, blk_b = ((uint64_t)a.Cout * a.sw) >> 4;
            uint32_t it = 0;
            int local = 0;
            for (int t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x, ++local) {
                const int acc = local & 1;
                const uint32_t use = (uint32_t)local >> 1;
                if (!tma::mbar_wait(&tempty[acc], (use & 1u) ^ 1u)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t d = tmem + (uint32_t)(acc * a.Cout);
                for (int kk = 0; kk < nk; ++kk, ++it) {
                    const int s = (int)(it % (uint32_t)a.stages);
                    if (!tma::mbar_wait(&full[s], (it / (uint32_t)a.stages) & 1u)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint64_t da = d0 + (uint64_t)s * (a.stage_bytes >> 4), db = da + (a.a_bytes >> 4);
                    for (int b = 0; b < a.bps; ++b)
                        for (int k = 0; k < a.cb / 16; ++k)  // K step: 32 B along the swizzled row
                            mma(d, da + b * blk_a + 2 * k, db + b * blk_b + 2 * k, id, (kk | b | k) != 0);
                    commit(&empty[s]);
                }
                if (!ok) break;
                commit(&tfull[acc]);
            }
            // every MMA issued has completed before the TMEM is freed
            commit(&fin);
            if (!tma::mbar_wait(&fin, 0u)) ok = false;
        }
    } else {
        const int q = warp & 3;  // TMEM lane quarter this warp may read
        const int m = q * 32 + lane;
        int local = 0;
        for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++local) {
            const int acc = local & 1;
            if (!tma::mbar_wait(&tfull[acc], ((uint32_t)local >> 1) & 1u)) {
                ok = false;
                break;
            }
            fence_after();
            int n, x0, y0;
            conv_tile_origin(a, t, n, x0, y0);
            const int yy = y0 + m / a.bw, xx = x0 + m % a.bw;
            const bool valid = yy < a.H && xx < a.W;
            const long long p = ((long long)n * a.H + yy) * a.W + xx;
            const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * a.Cout);
            for (int c0 = 0; c0 < a.Cout; c0 += 8) {
                uint32_t r[8];
                tmem_ld8(base + (uint32_t)c0, r);
                if (!valid) continue;
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float x = __uint_as_float(r[j]);
                    if (a.bias) x += __ldg(a.bias + c0 + j);
                    if (a.relu) x = fmaxf(x, 0.0f);
                    v[j] = x;
                }
                if (a.out)
                    *reinterpret_cast<uint4*>(a.out + p * a.Cout + c0) =
                        make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                                   pack_bf16x2(v[6], v[7]));
                if (a.out32) {
                    float4* o = reinterpret_cast<float4*>(a.out32 + p * a.Cout + c0);
                    o[0] = make_float4(v[0], v[1], v[2], v[3]);
                    o[1] = make_float4(v[4], v[5], v[6], v[7]);
                }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) tma::mbar_arrive(&tempty[acc]);
        }
    }
    if (!ok) atomicExch(&g_nn_tma_err, 1);
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        tmem_free(tmem, a.ncols);
    }
}

// ------------------------------------------------------- weight gradient
struct WgradArgs {
    int Cin, Cout;
    int bw, tiles_x, tiles_y, ntiles, tiles_per_chunk;
    int cbo, swo, nbo;  // dout channel blocks: channels, row bytes, count
    int cbi, swi, nbi;  // input channel blocks
    int tpg, tps;       // taps per group (grid y); taps per MMA (tps x Cin <= 256)
    int stages;
    uint32_t stage_bytes, a_bytes, b_bytes;  // b_bytes: one tap's input box
    uint32_t a_lbo;                          // 0 when one block holds every output channel
    int ncols;
    float* partial;       // [chunk][co][tap][ci]
    float* bias_partial;  // [chunk][co], or null
};

__device__ __forceinline__ void wg_tile_origin(const WgradArgs& a, int t, int& n, int& x0, int& y0) {
    const int tx = t % a.tiles_x;
    const int r = t / a.tiles_x;
    x0 = tx * a.bw;
    y0 = (r % a.tiles_y) * (kWgK / a.bw);
    n = r / a.tiles_y;
}

__global__ void __launch_bounds__(kThreads, 1)
    wgrad_tma_kernel(const __grid_constant__ CUtensorMap m_in, const __grid_constant__ CUtensorMap m_dout,
                     const WgradArgs a) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = align1024(smem_raw);
    __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], done;
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int chunk = blockIdx.x;
    const int tap0 = blockIdx.y * a.tpg;
    const int ntap = a.tpg < 9 - tap0 ? a.tpg : 9 - tap0;
    const int t_begin = chunk * a.tiles_per_chunk;
    const int t_end = t_begin + a.tiles_per_chunk < a.ntiles ? t_begin + a.tiles_per_chunk : a.ntiles;
    const bool with_bias = a.bias_partial != nullptr && blockIdx.y == 0;
    // B operand of the bias gradient: 16 columns of ones (any layout of ones is ones)
    unsigned char* ones = smem + (size_t)a.stages * a.stage_bytes;
    for (int i = threadIdx.x; i < (int)(kOnesBytes / 4); i += kThreads)
        reinterpret_cast<uint32_t*>(ones)[i] = 0x3F803F80u;  // bf16 1.0 x 2
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");

    if (warp == 1) {
        tmem_alloc(&tmem_slot, a.ncols);
        fence_before();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < a.stages; ++s) {
            tma::mbar_init(&full[s], 1);
            tma::mbar_init(&empty[s], 1);
        }
        tma::mbar_init(&done, 1);
        tma::fence_barrier_init();
        tma::prefetch_map(&m_in);
        tma::prefetch_map(&m_dout);
    }
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            const uint32_t tx = (uint32_t)a.nbo * kWgK * a.swo + (uint32_t)ntap * a.b_bytes;
            uint32_t it = 0;
            for (int t = t_begin; t < t_end; ++t, ++it) {
                const int s = (int)(it % (uint32_t)a.stages);
                if (!tma::mbar_wait(&empty[s], ((it / (uint32_t)a.stages) & 1u) ^ 1u)) {
                    ok = false;
                    break;
                }
                int n, x0, y0;
                wg_tile_origin(a, t, n, x0, y0);
                unsigned char* A = smem + (size_t)s * a.stage_bytes;
                tma::mbar_arrive_expect_tx(&full[s], tx);
                for (int bo = 0; bo < a.nbo; ++bo)
                    tma::load_4d(A + (size_t)bo * kWgK * a.swo, &m_dout, bo * a.cbo, x0, y0, n, &full[s]);
                for (int j = 0; j < ntap; ++j) {
                    const int tap = tap0 + j;
                    unsigned char* B = A + a.a_bytes + (size_t)j * a.b_bytes;
                    for (int bi = 0; bi < a.nbi; ++bi)
                        tma::load_4d(B + (size_t)bi * kWgK * a.swi, &m_in, bi * a.cbi, x0 + tap % 3 - 1,
                                     y0 + tap / 3 - 1, n, &full[s]);
                }
            }
            for (int s = 0; s < a.stages; ++s)
                if ((uint32_t)s < it && !tma::mbar_wait(&full[s], ((it - 1 - s) / (uint32_t)a.stages) & 1u)) ok = false;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t id_b = idesc(128, 16, true, true);
            // one MMA per group of tps taps (N = tps x Cin); the last group may be shorter
            const uint32_t id_full = idesc(128, a.tps * a.Cin, true, true);
            const uint32_t id_tail = idesc(128, (ntap - (ntap - 1) / a.tps * a.tps) * a.Cin, true, true);
            const uint32_t la = layout_of(a.swo), lb = layout_of(a.swi);
            const uint32_t sbo_a = 8u * (uint32_t)a.swo, sbo_b = 8u * (uint32_t)a.swi;
            const uint32_t lbo_b = (uint32_t)kWgK * (uint32_t)a.swi;
            const uint64_t d_ones = mdesc(saddr(ones), 128u, 256u, 0u);
            // stage 0's descriptors; a stage, K step and tap group are constant offsets
            const uint64_t da0 = mdesc(saddr(smem), a.a_lbo, sbo_a, la);
            const uint64_t db0 = mdesc(saddr(smem) + a.a_bytes, lbo_b, sbo_b, lb);
            const uint64_t k_a = (16u * (uint32_t)a.swo) >> 4, k_b = (16u * (uint32_t)a.swi) >> 4;
            const uint64_t grp_b = ((uint64_t)a.tps * a.b_bytes) >> 4;
            uint32_t it = 0;
            for (int t = t_begin; t < t_end; ++t, ++it) {
                const int s = (int)(it % (uint32_t)a.stages);
                if (!tma::mbar_wait(&full[s], (it / (uint32_t)a.stages) & 1u)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint64_t ds = (uint64_t)s * (a.stage_bytes >> 4);
                for (int k = 0; k < kWgK / 16; ++k) {
                    // K step: 16 pixels = two 8-row groups of each operand
                    const uint64_t da = da0 + ds + k * k_a;
                    const bool acc = (it | (uint32_t)k) != 0;
                    // the taps' input blocks are b_bytes = nbi x kWgK x swi apart, i.e. every
                    // cbi-channel block of the group sits lbo_b after the previous one: up to tps
                    // taps form one MMA with N = taps x Cin
                    for (int j = 0, g = 0; j < ntap; j += a.tps, ++g)
                        mma(tmem + (uint32_t)(j * a.Cin), da, db0 + ds + g * grp_b + k * k_b,
                            ntap - j < a.tps ? id_tail : id_full, acc);
                    if (with_bias) mma(tmem + (uint32_t)(ntap * a.Cin), da, d_ones, id_b, acc);
                }
                commit(&empty[s]);
            }
            commit(&done);
            if (!tma::mbar_wait(&done, 0u)) ok = false;
        }
    } else {
        const int q = warp & 3;
        const int co = q * 32 + lane;  // TMEM lane = output channel
        if (!tma::mbar_wait(&done, 0u)) ok = false;
        fence_after();
        const uint32_t base = tmem + ((uint32_t)(q * 32) << 16);
        for (int j = 0; j < ntap; ++j) {
            float* dst = a.partial + (((size_t)chunk * a.Cout + (co < a.Cout ? co : 0)) * 9 + tap0 + j) * a.Cin;
            for (int c0 = 0; c0 < a.Cin; c0 += 8) {
                uint32_t r[8];
                tmem_ld8(base + (uint32_t)(j * a.Cin + c0), r);
                if (co >= a.Cout) continue;
                float4* o = reinterpret_cast<float4*>(dst + c0);
                o[0] = make_float4(__uint_as_float(r[0]), __uint_as_float(r[1]), __uint_as_float(r[2]),
                                   __uint_as_float(r[3]));
                o[1] = make_float4(__uint_as_float(r[4]), __uint_as_float(r[5]), __uint_as_float(r[6]),
                                   __uint_as_float(r[7]));
            }
        }
        if (with_bias) {
            uint32_t r[8];
            tmem_ld8(base + (uint32_t)(ntap * a.Cin), r);
            if (co < a.Cout) a.bias_partial[(size_t)chunk * a.Cout + co] = __uint_as_float(r[0]);
        }
    }
    if (!ok) atomicExch(&g_nn_tma_err, 1);
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        tmem_free(tmem, a.ncols);
    }
}

// ------------------------------------------------------------ halo kernels
// A tile is 8 pixels wide and 16 rows tall (128 pixels).  Its input plus a
// one-pixel border (10 x 18 pixels) comes in once per tile, one 4-D TMA box
// per 8-channel plane, in the canonical no-swizzle layout: plane j holds
// [18 rows][10 pixels][8 channels], 16 bytes a pixel.  Every tap reads the
// same planes from a shifted start: the 8 pixels of a tile row are one core
// matrix, tile rows are one halo row (160 B) apart, planes kHaloPlane apart.
// Nine taps thus cost one load per plane instead of nine, and no MMA row is
// wasted (8-pixel tile rows never wrap inside a core matrix).
constexpr int kHx = 8, kHy = 16;
constexpr int kHaloW = kHx + 2, kHaloH = kHy + 2;
constexpr uint32_t kHaloBox = kHaloW * kHaloH * 16;  // 2880 B
constexpr uint32_t kHaloPlane = 2944;                // the box rounded up to 128 B
constexpr uint32_t kHaloRow = kHaloW * 16;           // 160 B

__device__ __forceinline__ void halo_tile_origin(int tiles_x, int tiles_y, int t, int& n, int& x0, int& y0) {
    const int tx = t % tiles_x;
    const int r = t / tiles_x;
    x0 = tx * kHx;
    y0 = (r % tiles_y) * kHy;
    n = r / tiles_y;
}

// shared-memory offset of tap `tap`'s first pixel in a halo plane
__device__ __forceinline__ uint32_t tap_offset(int tap) { return (uint32_t)((tap / 3) * kHaloW + tap % 3) * 16u; }

struct HaloConvArgs {
    int H, W, Cin, Cout;
    int tiles_x, tiles_y, ntiles;
    int planes;  // Cin / 8
    int stages;
    uint32_t stage_bytes, w_bytes;  // one tile's planes; the resident weights (rounded to 1024)
    int ncols;
    const __nv_bfloat16* w;  // [Cout][9][Cin]
    const float* bias;
    int relu;
    __nv_bfloat16* out;
    float* out32;
};

// Convolution with the weights resident in shared memory: [tap][ci / 8][co][8]
// (K-major B: core matrices of 8 output channels x 16 B, 128 B apart; the
// next 8 input channels Cout x 16 B further).
__global__ void __launch_bounds__(kThreads, 1)
    conv3x3_halo_kernel(const __grid_constant__ CUtensorMap m_in, const HaloConvArgs a) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = align1024(smem_raw);
    unsigned char* ring = smem + a.w_bytes;
    __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], tfull[2], tempty[2], fin;
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kc = a.Cin / 8;

    for (int e = threadIdx.x; e < 9 * kc * a.Cout; e += kThreads) {
        const int co = e % a.Cout, r = e / a.Cout;
        const int j = r % kc, tap = r / kc;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(a.w + ((size_t)co * 9 + tap) * a.Cin + 8 * j));
        *reinterpret_cast<uint4*>(smem + ((size_t)r * a.Cout + co) * 16) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the tensor cores read them
    if (warp == 1) {
        tmem_alloc(&tmem_slot, a.ncols);
        fence_before();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < a.stages; ++s) {
            tma::mbar_init(&full[s], 1);
            tma::mbar_init(&empty[s], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tma::mbar_init(&tfull[i], 1);
            tma::mbar_init(&tempty[i], 4);
        }
        tma::mbar_init(&fin, 1);
        tma::fence_barrier_init();
        tma::prefetch_map(&m_in);
    }
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            const uint32_t tx = (uint32_t)a.planes * kHaloBox;
            int s = 0;
            uint32_t ph = 0, used = 0;
            for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
                if (!tma::mbar_wait(&empty[s], ph ^ 1u)) {
                    ok = false;
                    break;
                }
                int n, x0, y0;
                halo_tile_origin(a.tiles_x, a.tiles_y, t, n, x0, y0);
                unsigned char* st = ring + (size_t)s * a.stage_bytes;
                tma::mbar_arrive_expect_tx(&full[s], tx);
                for (int j = 0; j < a.planes; ++j)
                    tma::load_4d(st + (size_t)j * kHaloPlane, &m_in, 8 * j, x0 - 1, y0 - 1, n, &full[s]);
                ++used;
                if (++s == a.stages) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            // the last fill of every stage has landed before the CTA can exit
            for (int q = 0; q < a.stages; ++q)
                if ((uint32_t)q < used && !tma::mbar_wait(&full[q], ((used - 1 - q) / (uint32_t)a.stages) & 1u))
                    ok = false;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t id = idesc(kConvM, a.Cout, false, false);
            // descriptors built once: one thread's dependent integer chain per
            // descriptor costs more than the MMA it feeds, so a tap's operands are
            // a base plus constant offsets (16-byte units)
            const uint32_t wstep = (uint32_t)a.Cout * 16u;
            const uint64_t dw0 = mdesc(saddr(smem), wstep, 128u, 0u);
            const uint64_t dh0 = mdesc(saddr(ring), kHaloPlane, kHaloRow, 0u);
            const uint64_t tap_w = ((uint64_t)kc * wstep) >> 4, k_w = (2u * wstep) >> 4, k_h = (2u * kHaloPlane) >> 4;
            int s = 0, local = 0;
            uint32_t ph = 0;
            for (int t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x, ++local) {
                const int acc = local & 1;
                if (!tma::mbar_wait(&tempty[acc], (((uint32_t)local >> 1) & 1u) ^ 1u) ||
                    !tma::mbar_wait(&full[s], ph)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t d = tmem + (uint32_t)(acc * a.Cout);
                const uint64_t dh = dh0 + (uint64_t)s * (a.stage_bytes >> 4);
#pragma unroll
                for (int tap = 0; tap < 9; ++tap) {
                    const uint64_t da = dh + (tap_offset(tap) >> 4), db = dw0 + (uint64_t)tap * tap_w;
                    mma(d, da, db, id, tap != 0);
                    // K steps 1..: planes 2k, 2k + 1
                    for (int k = 1; k < kc / 2; ++k) mma(d, da + k * k_h, db + k * k_w, id, true);
                }
                commit(&empty[s]);
                commit(&tfull[acc]);
                if (++s == a.stages) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            commit(&fin);
            if (!tma::mbar_wait(&fin, 0u)) ok = false;
        }
    } else {
        const int q = warp & 3;
        const int m = q * 32 + lane;
        int local = 0;
        for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++local) {
            const int acc = local & 1;
            if (!tma::mbar_wait(&tfull[acc], ((uint32_t)local >> 1) & 1u)) {
                ok = false;
                break;
            }
            fence_after();
            int n, x0, y0;
            halo_tile_origin(a.tiles_x, a.tiles_y, t, n, x0, y0);
            const int yy = y0 + m / kHx, xx = x0 + m % kHx;
            const bool valid = yy < a.H && xx < a.W;
            const long long p = ((long long)n * a.H + yy) * a.W + xx;
            const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * a.Cout);
            for (int c0 = 0; c0 < a.Cout; c0 += 8) {
                uint32_t r[8];
                tmem_ld8(base + (uint32_t)c0, r);
                if (!valid) continue;
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float x = __uint_as_float(r[j]);
                    if (a.bias) x += __ldg(a.bias + c0 + j);
                    if (a.relu) x = fmaxf(x, 0.0f);
                    v[j] = x;
                }
                if (a.out)
                    *reinterpret_cast<uint4*>(a.out + p * a.Cout + c0) =
                        make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                                   pack_bf16x2(v[6], v[7]));
                if (a.out32) {
                    float4* o = reinterpret_cast<float4*>(a.out32 + p * a.Cout + c0);
                    o[0] = make_float4(v[0], v[1], v[2], v[3]);
                    o[1] = make_float4(v[4], v[5], v[6], v[7]);
                }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) tma::mbar_arrive(&tempty[acc]);
        }
    }
    if (!ok) atomicExch(&g_nn_tma_err, 1);
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        tmem_free(tmem, a.ncols);
    }
}

}  // namespace

// ------------------------------------------------------------------- host
namespace {

constexpr int kSmTarget = 148;  // CTAs per launch of the weight gradient (one per SM)
constexpr size_t kOneCtaPerSm = 116 * 1024;  // dynamic shared memory that keeps a second CTA off the SM

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Channels per block: the widest of 64, 32, 16 that divides C (128-, 64- or
// 32-byte rows).
int channel_block(int C) { return C % 64 == 0 ? 64 : C % 32 == 0 ? 32 : 16; }

CUtensorMapSwizzle swizzle_of(int row_bytes) {
    return row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                            : row_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
}

// NHWC bf16 activations as the 4-D tensor (C, W, H, N), box (cb, bw, bh, 1);
// rows of 2 cb bytes swizzled to match (cb = 64, 32, 16), or not swizzled.
bool act_map(CUtensorMap* m, const void* base, int N, int H, int W, int C, int cb, int bw, int bh,
             bool swizzled = true) {
    auto enc = encoder();
    if (!enc) return false;
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {(cuuint32_t)cb, (cuuint32_t)bw, (cuuint32_t)bh, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, swizzled ? swizzle_of(2 * cb) : CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Weights [Cout][9][Cin] as the 3-D tensor (Cin, 9, Cout), box (cb, 1, Cout).
bool weight_map(CUtensorMap* m, const void* base, int Cin, int Cout, int cb) {
    auto enc = encoder();
    if (!enc) return false;
    cuuint64_t dims[3] = {(cuuint64_t)Cin, 9, (cuuint64_t)Cout};
    cuuint64_t strides[2] = {(cuuint64_t)Cin * 2, (cuuint64_t)Cin * 9 * 2};
    cuuint32_t box[3] = {(cuuint32_t)cb, 1, (cuuint32_t)Cout};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(2 * cb), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The input as (cb, W, H, N, C / cb): the channel blocks of a pixel as a fifth
// dimension (stride 2 cb bytes), box (cb, bw, bh, 1, bps) = bps blocks of
// 128 pixel rows back to back.
bool act_blocks_map(CUtensorMap* m, const void* base, int N, int H, int W, int C, int cb, int bw, int bh, int bps) {
    auto enc = encoder();
    if (!enc) return false;
    cuuint64_t dims[5] = {(cuuint64_t)cb, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N, (cuuint64_t)(C / cb)};
    cuuint64_t strides[4] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2, (cuuint64_t)cb * 2};
    cuuint32_t box[5] = {(cuuint32_t)cb, (cuuint32_t)bw, (cuuint32_t)bh, 1, (cuuint32_t)bps};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(2 * cb), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Weights [Cout][9][Cin] as (cb, Cout, 9, Cin / cb), box (cb, Cout, 1, bps).
bool weight_blocks_map(CUtensorMap* m, const void* base, int Cin, int Cout, int cb, int bps) {
    auto enc = encoder();
    if (!enc) return false;
    cuuint64_t dims[4] = {(cuuint64_t)cb, (cuuint64_t)Cout, 9, (cuuint64_t)(Cin / cb)};
    cuuint64_t strides[3] = {(cuuint64_t)Cin * 9 * 2, (cuuint64_t)Cin * 2, (cuuint64_t)cb * 2};
    cuuint32_t box[4] = {(cuuint32_t)cb, (cuuint32_t)Cout, 1, (cuuint32_t)bps};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(2 * cb), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Width of a box of `pixels` pixels (width x height = pixels, both powers of
// two, height <= 32) that pads the H x W image least; ties go to the wider box.
int box_width(int H, int W, int pixels) {
    long long best = -1;
    int pick = pixels;
    for (int bw = pixels; bw >= 4 && pixels / bw <= 32; bw /= 2) {
        const int bh = pixels / bw;
        const long long cost = (long long)((W + bw - 1) / bw) * bw * (long long)(((H + bh - 1) / bh) * bh);
        if (best < 0 || cost < best) {
            best = cost;
            pick = bw;
        }
    }
    return pick;
}

int tmem_columns(int need) {
    int n = 32;
    while (n < need) n *= 2;
    return n;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                                                       cudaSuccess || n < 1)
            n = kSmTarget;
    }
    return n;
}

// Largest dynamic shared memory the kernel may take, set for the current
// device on its first use there (function attributes are per device).
constexpr int kMaxDevices = 64;

template <typename K>
size_t max_dynamic_smem(K kernel, size_t (&per_device)[kMaxDevices]) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    if (per_device[dev] != 0) return per_device[dev];
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return 0;
    const size_t cap = 227 * 1024 - fa.sharedSizeBytes;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap) != cudaSuccess) return 0;
    return per_device[dev] = cap;
}

constexpr uint32_t kStageCap = 72 * 1024;  // bound of a weight-gradient stage and of a convolution stage of several channel blocks

struct WgPlan {
    WgradArgs a;
    int chunks, ngroups, bh;
};

// Tap groups, chunks and stages of the weight gradient; false for sizes the
// kernel does not take (Cout > 128).
bool wg_plan(int N, int H, int W, int Cin, int Cout, size_t smem_cap, WgPlan& p) {
    if (Cin % 16 || Cin > 256 || Cout % 16 || Cout > 128 || N < 1 || H < 1 || W < 1) return false;
    WgradArgs& a = p.a;
    a = WgradArgs{};
    a.Cin = Cin;
    a.Cout = Cout;
    a.cbo = channel_block(Cout);
    a.swo = 2 * a.cbo;
    a.nbo = Cout / a.cbo;
    a.cbi = channel_block(Cin);
    a.swi = 2 * a.cbi;
    a.nbi = Cin / a.cbi;
    // every tap of a group has Cin TMEM columns, the bias 16 more; a stage
    // (output-gradient box + one input box per tap) stays within kStageCap
    a.a_bytes = a.nbo == 1 ? (uint32_t)kWgK * a.swo : 128u * kWgK * 2u;
    a.b_bytes = (uint32_t)kWgK * Cin * 2u;
    int tpg = (512 - 16) / Cin;
    int by_smem = a.a_bytes < kStageCap ? (int)((kStageCap - a.a_bytes) / a.b_bytes) : 0;
    if (by_smem < 1) by_smem = 1;
    if (tpg > by_smem) tpg = by_smem;
    if (tpg > 9) tpg = 9;
    p.ngroups = (9 + tpg - 1) / tpg;
    a.tpg = (9 + p.ngroups - 1) / p.ngroups;
    a.tps = 256 / Cin < a.tpg ? 256 / Cin : a.tpg;
    a.bw = box_width(H, W, kWgK);
    p.bh = kWgK / a.bw;
    a.tiles_x = (W + a.bw - 1) / a.bw;
    a.tiles_y = (H + p.bh - 1) / p.bh;
    const long long nt = (long long)N * a.tiles_x * a.tiles_y;
    if (nt > (1LL << 30)) return false;
    a.ntiles = (int)nt;
    int chunks = kSmTarget / p.ngroups;
    if (chunks < 1) chunks = 1;
    if (chunks > a.ntiles) chunks = a.ntiles;
    a.tiles_per_chunk = (a.ntiles + chunks - 1) / chunks;
    p.chunks = (a.ntiles + a.tiles_per_chunk - 1) / a.tiles_per_chunk;  // every chunk non-empty
    // one dout block covering every output channel: the MMA's 128 rows all
    // read it (rows past Cout are never stored); else the blocks sit kWgK * swo
    // apart in a region of 128 rows
    a.a_lbo = a.nbo == 1 ? 0u : (uint32_t)kWgK * a.swo;
    a.stage_bytes = a.a_bytes + (uint32_t)a.tpg * a.b_bytes;
    const size_t budget = smem_cap > 1024 + kOnesBytes ? smem_cap - 1024 - kOnesBytes : 0;
    size_t st = budget / a.stage_bytes;
    if (st > (size_t)kMaxStages) st = kMaxStages;
    if (st < 2) return false;
    a.stages = (int)st;
    a.ncols = tmem_columns(a.tpg * Cin + 16);
    return a.ncols <= 512;
}

// Convolution over 8 x 16 tiles with resident weights: taken when the
// weights and two halo stages fit in shared memory, and either the weights are
// small or every CTA has at least two tiles to spread their load over.
bool halo_conv_plan(int N, int H, int W, int Cin, int Cout, size_t cap, HaloConvArgs& h) {
    h = HaloConvArgs{};
    h.H = H;
    h.W = W;
    h.Cin = Cin;
    h.Cout = Cout;
    h.tiles_x = (W + kHx - 1) / kHx;
    h.tiles_y = (H + kHy - 1) / kHy;
    const long long nt = (long long)N * h.tiles_x * h.tiles_y;
    if (nt > (1LL << 30)) return false;
    h.ntiles = (int)nt;
    h.planes = Cin / 8;
    h.stage_bytes = ((uint32_t)h.planes * kHaloPlane + 1023u) / 1024u * 1024u;
    h.w_bytes = ((uint32_t)(9 * Cin * Cout * 2) + 1023u) / 1024u * 1024u;
    if (h.w_bytes > 40 * 1024 && h.ntiles < 2 * kSmTarget) return false;
    if (cap < 1024 + (size_t)h.w_bytes + 2 * (size_t)h.stage_bytes) return false;
    size_t st = (cap - 1024 - h.w_bytes) / h.stage_bytes;
    if (st > (size_t)kMaxStages) st = kMaxStages;
    h.stages = (int)st;
    h.ncols = tmem_columns(2 * Cout);
    return true;
}

}  // namespace

int nn_conv3x3_tma(const void* in, int N, int H, int W, int Cin, const void* w, const float* bias, int Cout, int relu,
                   void* out, float* out32, cudaStream_t st) {
    if (Cin % 16 || Cin > 256 || Cout % 16 || Cout > 256 || N < 1 || H < 1 || W < 1) return -1;
    if (!aligned16(in) || !aligned16(w) || !aligned16(out) || !aligned16(out32)) return -1;
    static size_t hcaps[kMaxDevices] = {};
    const size_t hcap = max_dynamic_smem(conv3x3_halo_kernel, hcaps);
    if (hcap == 0) return -2;
    HaloConvArgs h;
    if (halo_conv_plan(N, H, W, Cin, Cout, hcap, h)) {
        h.w = static_cast<const __nv_bfloat16*>(w);
        h.bias = bias;
        h.relu = relu;
        h.out = static_cast<__nv_bfloat16*>(out);
        h.out32 = out32;
        CUtensorMap mh;
        if (!act_map(&mh, in, N, H, W, Cin, 8, kHaloW, kHaloH, false)) return -2;
        size_t dyn = 1024 + (size_t)h.w_bytes + (size_t)h.stages * h.stage_bytes;
        if (dyn < kOneCtaPerSm) dyn = kOneCtaPerSm;
        const int grid = h.ntiles < sm_count() ? h.ntiles : sm_count();
        conv3x3_halo_kernel<<<grid, kThreads, dyn, st>>>(mh, h);
        return cudaGetLastError() == cudaSuccess ? 0 : -2;
    }
    static size_t caps[kMaxDevices] = {};
    const size_t cap = max_dynamic_smem(conv3x3_tma_kernel, caps);
    if (cap == 0) return -2;
    ConvArgs a{};
    a.H = H;
    a.W = W;
    a.Cout = Cout;
    a.bw = box_width(H, W, kConvM);
    const int bh = kConvM / a.bw;
    a.tiles_x = (W + a.bw - 1) / a.bw;
    a.tiles_y = (H + bh - 1) / bh;
    const long long nt = (long long)N * a.tiles_x * a.tiles_y;
    if (nt > (1LL << 30)) return -1;
    a.ntiles = (int)nt;
    a.cb = channel_block(Cin);
    a.nkb = Cin / a.cb;
    a.sw = 2 * a.cb;
    // 128-byte rows: as many channel blocks per stage as divide the tap's and
    // keep the stage within kStageCap (each block's weights Cout x 128 B, a
    // multiple of the 1024-B swizzle span)
    a.bps = 1;
    if (a.cb == 64)
        for (int b = a.nkb; b > 1; --b)
            if (a.nkb % b == 0 && (uint32_t)b * (kConvM + Cout) * 128u <= kStageCap) {
                a.bps = b;
                break;
            }
    a.a_bytes = (uint32_t)a.bps * kConvM * a.sw;
    const uint32_t b_bytes = (uint32_t)(a.bps * Cout * a.sw);
    a.tx_bytes = a.a_bytes + b_bytes;
    a.stage_bytes = (a.tx_bytes + 1023u) / 1024u * 1024u;
    size_t stages = (cap - 1024) / a.stage_bytes;
    if (stages > (size_t)kMaxStages) stages = kMaxStages;
    if (stages < 2) return -1;
    a.stages = (int)stages;
    a.ncols = tmem_columns(2 * Cout);
    a.bias = bias;
    a.relu = relu;
    a.out = static_cast<__nv_bfloat16*>(out);
    a.out32 = out32;
    CUtensorMap mi, mw;
    if (a.bps > 1) {
        if (!act_blocks_map(&mi, in, N, H, W, Cin, a.cb, a.bw, bh, a.bps) ||
            !weight_blocks_map(&mw, w, Cin, Cout, a.cb, a.bps))
            return -2;
    } else if (!act_map(&mi, in, N, H, W, Cin, a.cb, a.bw, bh) || !weight_map(&mw, w, Cin, Cout, a.cb)) {
        return -2;
    }
    size_t dyn = (size_t)a.stages * a.stage_bytes + 1024;
    if (dyn < kOneCtaPerSm) dyn = kOneCtaPerSm;
    const int grid = a.ntiles < sm_count() ? a.ntiles : sm_count();
    conv3x3_tma_kernel<<<grid, kThreads, dyn, st>>>(mi, mw, a);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

size_t nn_wgrad_tma_partial_floats(int N, int H, int W, int Cin, int Cout) {
    WgPlan p;
    if (!wg_plan(N, H, W, Cin, Cout, 227 * 1024, p)) return 0;
    return (size_t)p.chunks * Cout * (9 * (size_t)Cin + 1);
}

int nn_wgrad_tma(const void* in, const void* dout, int N, int H, int W, int Cin, int Cout, float* partial, bool bias,
                 cudaStream_t st) {
    if (!aligned16(in) || !aligned16(dout) || !aligned16(partial)) return -1;
    static size_t caps[kMaxDevices] = {};
    const size_t cap = max_dynamic_smem(wgrad_tma_kernel, caps);
    if (cap == 0) return -2;
    WgPlan p;
    if (!wg_plan(N, H, W, Cin, Cout, cap, p)) return -1;
    WgradArgs a = p.a;
    a.partial = partial;
    a.bias_partial = bias ? partial + (size_t)p.chunks * Cout * 9 * Cin : nullptr;
    CUtensorMap mi, md;
    if (!act_map(&mi, in, N, H, W, Cin, a.cbi, a.bw, p.bh) || !act_map(&md, dout, N, H, W, Cout, a.cbo, a.bw, p.bh))
        return -2;
    size_t dyn = (size_t)a.stages * a.stage_bytes + kOnesBytes + 1024;
    if (dyn < kOneCtaPerSm) dyn = kOneCtaPerSm;
    wgrad_tma_kernel<<<dim3(p.chunks, p.ngroups), kThreads, dyn, st>>>(mi, md, a);
    return cudaGetLastError() == cudaSuccess ? p.chunks : -2;
}

int nn_tma_error(bool reset) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_nn_tma_err, sizeof(int)) != cudaSuccess) return -1;
    if (reset && v) {
        const int z = 0;
        cudaMemcpyToSymbol(g_nn_tma_err, &z, sizeof(int));
    }
    return v;
}

}  // namespace fwi
