// k_fwd_loop.cu — every forward time level of a batch in ONE cooperative launch.
//
// The per-tile work is the one-level pass of k_fwd_tma.cu (fwd_tile.cuh):
// compute_pressure + compute_seismogram of src/modeling/modeling.cu:301-353 in
// Jacobi order.  What changes is the time loop: instead of one launch per
// level, the persistent CTAs (all co-resident, guaranteed by the cooperative
// launch) loop over the levels themselves and meet at a grid barrier between
// levels, so a small survey whose fields stay in L2 is no longer bound by
// launch latency.  The producer warp keeps its TMA pipeline across levels
// (the stage / phase counters run on), the four field buffers rotate in the
// kernel, and the tensor maps of all four are kernel parameters.
//
// Grid barrier: after a CTA has written its tiles of a level, its first thread
// fences, increments a global counter and polls it (bounded, with a short
// sleep) until every CTA has arrived; the producer then issues a proxy fence so
// its next TMA reads see the other CTAs' stores.  A poll that gives up raises
// *err and the kernel returns with no copy in flight.  Waits give up after
// la.base.spin polls; the failure drill (la.base.stall) makes one CTA withhold
// the loads of its first tile, so its consumers' and then every other CTA's
// waits run out.
#include <cuda.h>
#include <cuda_runtime.h>

#include "fwd_tile.cuh"
#include "kargs.h"
#include "kernels.h"
#include "stencil.cuh"
#include "tma.cuh"

namespace fwi {

namespace {

using namespace ft;

// Gives up after `limit` polls, or when another CTA has raised *err (that CTA
// has left the level loop and will never arrive; checked every 32nd poll so
// that the flag's load does not slow the barrier).
__device__ __forceinline__ bool grid_barrier(unsigned* counter, unsigned target, uint32_t limit, const int* err) {
    __threadfence();
    atomicAdd(counter, 1u);
    for (uint32_t i = 0; i < limit; ++i) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(counter) : "memory");
        if (v >= target) return true;
        if ((i & 31u) == 31u && tma::ld_flag(err)) return false;  // every 32nd poll only
        __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// MINB: CTAs per SM the registers are budgeted for (shared memory permitting)
template <int TX, int S, bool ABC, int MINB>
__global__ void __launch_bounds__(kNT, MINB)
    fwd_loop_kernel(const __grid_constant__ FwdLoopMaps maps, const FwdLoopArgs la) {
    using G = Geom<1, TX>;
    extern __shared__ __align__(128) float smem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t empty[S];
    __shared__ TileMeta meta[S];
    __shared__ int abort_flag;
    const int tid = threadIdx.x;
    const FwdTmaArgs& b = la.base;
    const int total = __ldg(b.tile_base + b.ns);

    if (tid == 0) {
        for (int k = 0; k < S; ++k) {
            tma::mbar_init(&full[k], 1);
            tma::mbar_init(&empty[k], kNC / 32);
        }
        abort_flag = 0;
        tma::fence_barrier_init();
        tma::prefetch_map(&maps.vel);
    }
    __syncthreads();

    const int lane = tid & 31;
    int issued = 0;  // producer lane: loads issued so far (pipeline uses)
    int k = 0;       // pipeline use counter, continuous across levels
    int c = la.buf_cur, o = la.buf_old, f = la.buf_free;
    for (int t = la.t_begin; t < la.t_end; ++t) {
        FwdTmaArgs a = b;
        a.sample1 = (t + 1 < la.nt) ? t + 1 : -1;
        a.sample2 = -1;
        a.rec_sample0 = (la.record && t > la.tlag) ? t - la.tlag : -1;
        a.rec_sample1 = -1;
        a.out1 = la.bufs[f];
        a.out2 = nullptr;
        bool ok = true;
        if (tid >= kNC) {
            // ---------- producer: lane 0 issues this level's tiles
            if (lane == 0) {
                fence_proxy_async_global();
                int kk = k;
                for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++kk) {
                    const int stg = kk % S;
                    if (kk >= S && !tma::mbar_wait(&empty[stg], (uint32_t)(((kk / S) - 1) & 1), b.spin)) {
                        ok = false;
                        break;
                    }
                    if (b.stall == (int)blockIdx.x && t == la.t_begin && kk == k) continue;  // failure drill
                    const TileInfo ti = decode(a, tile, TX);
                    const ShotDesc sd = a.shots[ti.s];
                    TileMeta& mt = meta[stg];
                    mt.s = ti.s;
                    mt.x0 = ti.x0;
                    mt.z0 = ti.z0;
                    mt.nxx = sd.nxx;
                    mt.col_off = sd.col_off;
                    mt.has_src = a.sample1 >= 0 &&
                                 st::has_points(a.inj, sd.col_off, ti.x0, min(ti.x0 + TX, sd.nxx));
                    mt.rec_kb = mt.rec_ke = 0;  // receivers are recorded at the end of the level
                    float* base = smem + stg * G::STAGE;
                    tma::mbar_arrive_expect_tx(&full[stg], G::BYTES);
                    tma::load_3d(base, &maps.cur[c], ti.z0 - 4, ti.x0 - 4, ti.s, &full[stg]);
                    tma::load_3d(base + G::CUR, &maps.pt[o], ti.z0, ti.x0, ti.s, &full[stg]);
                    tma::load_3d(base + G::CUR + G::PTW, &maps.vel, ti.z0, ti.x0 + sd.vel_col,
                                 a.vel_shared ? 0 : ti.s, &full[stg]);
                    issued = kk + 1;
                }
                if (!ok) {
                    atomicExch(a.err, 1);
                    abort_flag = 1;
                }
            }
        } else {
            // ---------- consumers
            int kk = k;
            for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++kk) {
                const int stg = kk % S;
                if (!tma::mbar_wait(&full[stg], (uint32_t)((kk / S) & 1), b.spin)) {
                    if (lane == 0) atomicExch(a.err, 1);
                    abort_flag = 1;
                    ok = false;
                    break;
                }
                const TileMeta mt = meta[stg];
                Tile tl;
                tl.ti.s = mt.s;
                tl.ti.x0 = mt.x0;
                tl.ti.z0 = mt.z0;
                tl.nxx = mt.nxx;
                tl.col_off = mt.col_off;
                tl.cur = smem + stg * G::STAGE;
                tl.old = tl.cur + G::CUR;
                tl.vel = tl.old + G::PTW;
                tl.mid = nullptr;
                tl.has_src = mt.has_src != 0;
                const float* b1d = ABC ? a.b1d : nullptr;
                const bool inner = st::tile_inner(tl.ti.z0, kTZ, tl.ti.x0, TX, a.nzz, tl.nxx);
                const bool undamped = st::tile_undamped(b1d, a.nb, tl.ti.z0, kTZ, tl.ti.x0, TX, a.nzz, tl.nxx);
                if (inner && undamped) final_pass<1, TX, false, false>(a, tl);
                else if (inner) final_pass<1, TX, ABC, false>(a, tl);
                else final_pass<1, TX, ABC, true>(a, tl);
                __syncwarp();
                if (lane == 0) tma::mbar_arrive(&empty[stg]);
            }
        }
        // the CTA's tiles of level t are written; its receivers record Q^t,
        // which stays in buffer c until level t + 2 writes there (the damper
        // of the absorbing boundary as in compute_seismogram's ABC run);
        // then the grid barrier
        if (la.record && t > la.tlag && b.seis) {
            const float* qt = la.bufs[c];
            const int r1 = __ldg(la.rec_cta_ptr + blockIdx.x + 1);
            for (int r = __ldg(la.rec_cta_ptr + blockIdx.x) + tid; r < r1; r += kNT) {
                const RecPoint rp = la.rec_pts[r];
                const float d = ABC ? st::damp(st::rows_info(b.b1d, b.nb, rp.z, b.nzz),
                                               st::col_info(b.b1d, b.nb, rp.x, rp.nxx), 0)
                                    : 1.0f;
                b.seis[rp.soff + (t - la.tlag)] = d * __ldcg(qt + rp.g);
            }
        }
        __syncthreads();
        if (tid == 0 && !abort_flag) {
            if (!grid_barrier(la.sync, (unsigned)(t - la.t_begin + 1) * gridDim.x, b.spin, b.err)) {
                atomicExch(b.err, 1);
                abort_flag = 1;
            }
        }
        __syncthreads();
        if (abort_flag) {
            // never leave copies in flight behind an exiting CTA: wait (bounded)
            // for the last S loads issued; phases already consumed pass at once
            if (tid == kNC)
                for (int q = (issued > S ? issued - S : 0); q < issued; ++q)
                    tma::mbar_wait(&full[q % S], (uint32_t)((q / S) & 1), b.spin);
            return;
        }
        // this CTA's tile count per level is fixed: advance the pipeline counter
        for (int tile = blockIdx.x; tile < total; tile += gridDim.x) ++k;
        const int po = o;
        o = c;
        c = f;
        f = po;
    }
}

template <int TX, int S>
constexpr size_t loop_smem() {
    return (size_t)S * Geom<1, TX>::STAGE * sizeof(float);
}

template <int TX, int S, bool ABC, int B>
cudaError_t loop_configure_one(int* ctas) {
    auto fn = fwd_loop_kernel<TX, S, ABC, B>;
    const size_t smem = loop_smem<TX, S>();
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, kNT, smem);
}

template <int TX, int S, int B>
cudaError_t loop_configure(int* ctas) {
    int a = 0, b = 0;
    cudaError_t e = loop_configure_one<TX, S, true, B>(&a);
    if (e == cudaSuccess) e = loop_configure_one<TX, S, false, B>(&b);
    *ctas = a < b ? a : b;
    return e;
}

template <int TX, int S, int B>
cudaError_t loop_launch(const FwdLoopMaps& maps, const FwdLoopArgs& la, int grid, cudaStream_t st) {
    const size_t smem = loop_smem<TX, S>();
    void* args[] = {const_cast<FwdLoopMaps*>(&maps), const_cast<FwdLoopArgs*>(&la)};
    if (la.base.b1d)
        return cudaLaunchCooperativeKernel((const void*)fwd_loop_kernel<TX, S, true, B>, dim3(grid), dim3(kNT), args,
                                           smem, st);
    return cudaLaunchCooperativeKernel((const void*)fwd_loop_kernel<TX, S, false, B>, dim3(grid), dim3(kNT), args,
                                       smem, st);
}

// (tile columns, pipeline stages, CTAs per SM of the register budget).  Measured
// on the B200: 3 CTAs per SM (70 registers) beat 2 for 16-column tiles on
// HBM-bound surveys; 8-column tiles at 3-4 CTAs per SM lost everywhere (halo
// overhead, a costlier grid barrier) and are not built.
#define FWI_FWD_LOOP_VARIANTS(X) X(32, 2, 2) X(16, 3, 2) X(16, 2, 2) X(16, 2, 3)

}  // namespace

bool fwd_loop_supported(int TX, int S, int B) {
#define FWI_X(tx, s, b) if (TX == tx && S == s && B == b) return true;
    FWI_FWD_LOOP_VARIANTS(FWI_X)
#undef FWI_X
    return false;
}

cudaError_t fwd_loop_configure(int* ctas_per_sm, int TX, int S, int B) {
#define FWI_X(tx, s, b) if (TX == tx && S == s && B == b) return loop_configure<tx, s, b>(ctas_per_sm);
    FWI_FWD_LOOP_VARIANTS(FWI_X)
#undef FWI_X
    return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_loop(int TX, int S, int B, const FwdLoopMaps& maps, const FwdLoopArgs& la, int grid,
                            cudaStream_t st) {
#define FWI_X(tx, s, b) if (TX == tx && S == s && B == b) return loop_launch<tx, s, b>(maps, la, grid, st);
    FWI_FWD_LOOP_VARIANTS(FWI_X)
#undef FWI_X
    return cudaErrorInvalidValue;
}

}  // namespace fwi
