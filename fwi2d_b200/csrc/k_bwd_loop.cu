// k_bwd_loop.cu — every back-propagation level of a batch in ONE cooperative launch.
//
// Per level and point this is the backward step of k_stencil.cu
// (inject_seismogram / inject_adjoint + cross_correlation / build_gradient,
// migration.cu:117-180, inversion.cu:381-444), with the same arithmetic
// (st::bwd_update4): the source field steps back through the random boundary,
// the receiver field forward with the receiver traces injected, and the image
// or gradient and the source illumination accumulate per shot.  It moves
// 44 B per point and level (7 fields read, 4 written), so the layout is built
// for memory-level parallelism:
//
//   * persistent CTAs (one per SM, all co-resident through the cooperative
//     launch) own a fixed set of 128 x TX tiles and loop over the levels,
//     meeting at a bounded grid barrier between levels (as k_fwd_loop.cu);
//   * one producer warp streams every tile's seven inputs into an S-stage
//     shared-memory ring with TMA: the two fields read through the stencil
//     with their 4-cell halo, the five read pointwise without (velocity,
//     source and receiver fields of the level before, both accumulators);
//   * eight consumer warps compute from shared memory (thread = 4 rows of
//     TX/8 columns, register-window Laplacians) and store the four outputs
//     with coalesced float4 stores, then release the stage;
//   * the receivers' samples are injected after a CTA's tiles of the level
//     are stored and before the grid barrier: the host lists, per CTA, the
//     receiver points of its tiles (a CTA owns the same tiles at every
//     level), and its threads add each point's samples with one
//     read-modify-write, so no tile load or update waits on the receiver
//     tables.
//
// Every wait is bounded (tma::kSpinLimit polls); a wait that gives up raises
// *err and the kernel returns once its own copies in flight have landed.
// Failure drill: the DRILL instantiations take the limit from a.spin, give a
// grid-barrier poll up once *err is raised, and let CTA a.stall withhold the
// loads of its first tile, so its consumers' and then every other CTA's waits
// run out.  Only contexts given the test keys launch them; the production
// instantiations keep the constant limit (whose code the kernel was measured
// with: even a run-time limit changes the schedule).
#include <cuda.h>
#include <cuda_runtime.h>

#include "fwd_tile.cuh"
#include "kargs.h"
#include "kernels.h"
#include "stencil.cuh"
#include "tma.cuh"

namespace fwi {

namespace {

using ft::kNC;
using ft::kNT;
using ft::kTZ;

template <int TX>
struct BGeom {
    static constexpr int CZ = kTZ + 8;            // rows of a stencil tile
    static constexpr int CX = TX + 8;             // columns of a stencil tile
    static constexpr int ST = CZ * CX;            // floats of a stencil tile
    static constexpr int PT = kTZ * TX;           // floats of a pointwise tile
    static constexpr int STAGE = 2 * ST + 5 * PT; // ps_st, pr_st | vel, ps, pr, acc_a, acc_b
    static constexpr uint32_t BYTES = STAGE * 4;
    static_assert((ST * 4) % 128 == 0 && (PT * 4) % 128 == 0, "TMA destinations must stay 128-byte aligned");
    static_assert(CZ <= 256 && CX <= 256, "TMA box extent");
};

struct BMeta {
    int s, x0, z0, nxx, col_off;
};

// Gives up after `limit` polls; the drill instantiation also gives up when
// another CTA has raised *err (that CTA has left the level loop and will
// never arrive; checked every 32nd poll).
template <bool DRILL>
__device__ __forceinline__ bool grid_barrier(unsigned* counter, unsigned target, uint32_t limit, const int* err) {
    __threadfence();
    atomicAdd(counter, 1u);
    for (uint32_t i = 0; i < limit; ++i) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(counter) : "memory");
        if (v >= target) return true;
        if (DRILL && (i & 31u) == 31u && tma::ld_flag(err)) return false;
        __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Tile -> (shot, first row, first column): tiles run down the columns of a
// shot first, shots follow each other (tile_base: prefix sums per shot).
__device__ __forceinline__ ft::TileInfo decode_tile(const BwdLoopArgs& a, int tile, int tx) {
    int lo = 0, hi = a.ns;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(a.tile_base + mid) <= tile) lo = mid;
        else hi = mid;
    }
    const int local = tile - __ldg(a.tile_base + lo);
    ft::TileInfo ti;
    ti.s = lo;
    ti.z0 = (local % a.ntz) * kTZ;
    ti.x0 = (local / a.ntz) * tx;
    return ti;
}

// Consumer pass over one staged tile of level b.
template <int TX, bool GRAD, bool EDGE>
__device__ __forceinline__ void bwd_tile(const BwdLoopArgs& a, const float* stage, const BMeta& mt,
                                         float* ps_out, float* pr_out) {
    using G = BGeom<TX>;
    constexpr int CPW = TX / 8;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int z = mt.z0 + 4 * lane;
    if (z >= a.ldz) return;
    const float* t_ps = stage;
    const float* t_pr = stage + G::ST;
    const float* t_v = stage + 2 * G::ST;
    const float* t_ps_o = t_v + G::PT;
    const float* t_pr_o = t_v + 2 * G::PT;
    const float* t_a = t_v + 3 * G::PT;
    const float* t_b = t_v + 4 * G::PT;
    const st::Rows rows = st::rows_info(nullptr, 0, z, a.nzz);
    const int c0 = warp * CPW;
    float ls[CPW][4], lr[CPW][4];
    float4 psold[CPW], pr[CPW];
    st::lap_run<G::CZ, CPW>(t_ps, 4 * lane + 4, c0 + 4, ls, psold);
    st::lap_run<G::CZ, CPW>(t_pr, 4 * lane + 4, c0 + 4, lr, pr);
    const size_t so = (size_t)mt.s * a.fstride;
#pragma unroll
    for (int m = 0; m < CPW; ++m) {
        const int c = c0 + m;
        const int gx = mt.x0 + c;
        if (gx >= mt.nxx) break;
        const int po = c * kTZ + 4 * lane;
        const float4 vv = *reinterpret_cast<const float4*>(t_v + po);
        const float4 ps = *reinterpret_cast<const float4*>(t_ps_o + po);
        const float4 prold = *reinterpret_cast<const float4*>(t_pr_o + po);
        const float4 ga = *reinterpret_cast<const float4*>(t_a + po);
        const float4 gb = *reinterpret_cast<const float4*>(t_b + po);
        const bool colok = !EDGE || (gx >= 4 && gx < mt.nxx - 4);
        const st::Bwd4 r = st::bwd_update4<GRAD, EDGE>(ls[m], psold[m], lr[m], pr[m], ps, prold, vv, ga, gb,
                                                       a.dt2idh2, a.dt, a.idh2, rows, colok);
        const float4 rv = r.pr;  // the receivers' samples are added at the end of the level
        const size_t g = so + (size_t)gx * a.ldz + z;
        *reinterpret_cast<float4*>(ps_out + g) = r.ps;
        *reinterpret_cast<float4*>(pr_out + g) = rv;
        *reinterpret_cast<float4*>(a.acc_a + g) = r.a;
        *reinterpret_cast<float4*>(a.acc_b + g) = r.b;
    }
}

template <int TX, int S, bool GRAD, bool DRILL>
__global__ void __launch_bounds__(kNT, TX == 8 ? 2 : 1)
    bwd_loop_kernel(const __grid_constant__ BwdLoopMaps maps, const BwdLoopArgs a) {
    using G = BGeom<TX>;
    extern __shared__ __align__(128) float smem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t empty[S];
    __shared__ BMeta meta[S];
    __shared__ int abort_flag;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int total = __ldg(a.tile_base + a.ns);

    if (tid == 0) {
        for (int k = 0; k < S; ++k) {
            tma::mbar_init(&full[k], 1);
            tma::mbar_init(&empty[k], kNC / 32);
        }
        abort_flag = 0;
        tma::fence_barrier_init();
        tma::prefetch_map(&maps.vel);
        tma::prefetch_map(&maps.acc_a);
        tma::prefetch_map(&maps.acc_b);
    }
    __syncthreads();

    const uint32_t limit = DRILL ? a.spin : tma::kSpinLimit;
    int issued = 0;  // producer lane: loads issued so far
    int k = 0;       // pipeline use counter, continuous across levels
    for (int b = a.b_begin; b < a.b_end; ++b) {
        const int p = b & 1;
        const int sample = (b + 1 < a.nt) ? a.nt - 1 - (b + 1) : -1;
        bool ok = true;
        if (tid >= kNC) {
            // ---------- producer: lane 0 streams this level's tiles
            if (lane == 0) {
                fence_proxy_async_global();
                int kk = k;
                for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++kk) {
                    const int stg = kk % S;
                    if (kk >= S && !tma::mbar_wait(&empty[stg], (uint32_t)(((kk / S) - 1) & 1), limit)) {
                        ok = false;
                        break;
                    }
                    if (DRILL && a.stall == (int)blockIdx.x && b == a.b_begin && kk == k) continue;  // the drill
                    const ft::TileInfo ti = decode_tile(a, tile, TX);
                    const int s = ti.s, z0 = ti.z0, x0 = ti.x0;
                    const ShotDesc sd = a.shots[s];
                    BMeta& mt = meta[stg];
                    mt.s = s;
                    mt.x0 = x0;
                    mt.z0 = z0;
                    mt.nxx = sd.nxx;
                    mt.col_off = sd.col_off;
                    float* base = smem + stg * G::STAGE;
                    float* pts = base + 2 * G::ST;
                    tma::mbar_arrive_expect_tx(&full[stg], G::BYTES);
                    tma::load_3d(base, &maps.ps_st[p], z0 - 4, x0 - 4, s, &full[stg]);
                    tma::load_3d(base + G::ST, &maps.pr_st[p], z0 - 4, x0 - 4, s, &full[stg]);
                    tma::load_3d(pts, &maps.vel, z0, x0 + sd.vel_col, a.vel_shared ? 0 : s, &full[stg]);
                    tma::load_3d(pts + G::PT, &maps.ps_pt[p], z0, x0, s, &full[stg]);
                    tma::load_3d(pts + 2 * G::PT, &maps.pr_pt[p], z0, x0, s, &full[stg]);
                    tma::load_3d(pts + 3 * G::PT, &maps.acc_a, z0, x0, s, &full[stg]);
                    tma::load_3d(pts + 4 * G::PT, &maps.acc_b, z0, x0, s, &full[stg]);
                    issued = kk + 1;
                }
                if (!ok) {
                    atomicExch(a.err, 1);
                    abort_flag = 1;
                }
            }
        } else {
            // ---------- consumers
            float* ps_out = a.ps[p];
            float* pr_out = a.pr[p ^ 1];
            int kk = k;
            for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++kk) {
                const int stg = kk % S;
                if (!tma::mbar_wait(&full[stg], (uint32_t)((kk / S) & 1), limit)) {
                    if (lane == 0) atomicExch(a.err, 1);
                    abort_flag = 1;
                    ok = false;
                    break;
                }
                const BMeta mt = meta[stg];
                const float* stage = smem + stg * G::STAGE;
                if (st::tile_inner(mt.z0, kTZ, mt.x0, TX, a.nzz, mt.nxx))
                    bwd_tile<TX, GRAD, false>(a, stage, mt, ps_out, pr_out);
                else
                    bwd_tile<TX, GRAD, true>(a, stage, mt, ps_out, pr_out);
                __syncwarp();
                if (lane == 0) tma::mbar_arrive(&empty[stg]);
            }
        }
        // the CTA's tiles of level b are written: the receiver points in them
        // take this level's samples (one read-modify-write per point, its
        // receivers in entry order), then the grid barrier
        __syncthreads();
        if (sample >= 0) {
            float* pr_out = a.pr[p ^ 1];
            const int q1 = __ldg(a.inj_cta_ptr + blockIdx.x + 1);
            for (int q = __ldg(a.inj_cta_ptr + blockIdx.x) + tid; q < q1; q += kNT) {
                const InjPoint pt = a.inj_pts[q];
                float v = pr_out[pt.g];
                for (int e = pt.e0; e < pt.e1; ++e) {
                    const float amp = a.inj.scale * __ldg(a.inj.series + __ldg(a.inj_soff + e) + sample);
                    v += amp;
                }
                pr_out[pt.g] = v;
            }
            __syncthreads();
        }
        if (tid == 0 && !abort_flag) {
            if (!grid_barrier<DRILL>(a.sync, (unsigned)(b - a.b_begin + 1) * gridDim.x, limit, a.err)) {
                atomicExch(a.err, 1);
                abort_flag = 1;
            }
        }
        __syncthreads();
        if (abort_flag) {
            // never leave copies in flight behind an exiting CTA
            if (tid == kNC)
                for (int q = (issued > S ? issued - S : 0); q < issued; ++q)
                    tma::mbar_wait(&full[q % S], (uint32_t)((q / S) & 1), limit);
            return;
        }
        for (int tile = blockIdx.x; tile < total; tile += gridDim.x) ++k;
    }
}

template <int TX, int S>
constexpr size_t bwd_smem() {
    return (size_t)S * BGeom<TX>::STAGE * sizeof(float);
}

template <int TX, int S, bool GRAD>
cudaError_t bwd_configure_one(int* ctas) {
    auto fn = bwd_loop_kernel<TX, S, GRAD, false>;
    const size_t smem = bwd_smem<TX, S>();
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(bwd_loop_kernel<TX, S, GRAD, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, kNT, smem);
}

template <int TX, int S>
cudaError_t bwd_configure(int* ctas) {
    int x = 0, y = 0;
    cudaError_t e = bwd_configure_one<TX, S, true>(&x);
    if (e == cudaSuccess) e = bwd_configure_one<TX, S, false>(&y);
    *ctas = x < y ? x : y;
    return e;
}

template <int TX, int S>
cudaError_t bwd_launch(bool gradient, const BwdLoopMaps& maps, const BwdLoopArgs& la, int grid, cudaStream_t st) {
    const size_t smem = bwd_smem<TX, S>();
    void* args[] = {const_cast<BwdLoopMaps*>(&maps), const_cast<BwdLoopArgs*>(&la)};
    const bool drill = la.stall >= 0 || la.spin != tma::kSpinLimit;
    const void* fn = gradient ? (drill ? (const void*)bwd_loop_kernel<TX, S, true, true>
                                       : (const void*)bwd_loop_kernel<TX, S, true, false>)
                              : (drill ? (const void*)bwd_loop_kernel<TX, S, false, true>
                                       : (const void*)bwd_loop_kernel<TX, S, false, false>);
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kNT), args, smem, st);
}

#define FWI_BWD_LOOP_VARIANTS(X) X(16, 3) X(16, 2) X(8, 4) X(8, 3)

}  // namespace

bool bwd_loop_supported(int TX, int S) {
#define FWI_X(tx, s) if (TX == tx && S == s) return true;
    FWI_BWD_LOOP_VARIANTS(FWI_X)
#undef FWI_X
    return false;
}

cudaError_t bwd_loop_configure(int* ctas_per_sm, int TX, int S) {
#define FWI_X(tx, s) if (TX == tx && S == s) return bwd_configure<tx, s>(ctas_per_sm);
    FWI_BWD_LOOP_VARIANTS(FWI_X)
#undef FWI_X
    return cudaErrorInvalidValue;
}

cudaError_t launch_bwd_loop(int TX, int S, bool gradient, const BwdLoopMaps& maps, const BwdLoopArgs& la, int grid,
                            cudaStream_t st) {
#define FWI_X(tx, s) if (TX == tx && S == s) return bwd_launch<tx, s>(gradient, maps, la, grid, st);
    FWI_BWD_LOOP_VARIANTS(FWI_X)
#undef FWI_X
    return cudaErrorInvalidValue;
}

}  // namespace fwi
