// k_fwd_tma.cu — forward leapfrog steps with TMA-staged tiles in a persistent,
// pipelined kernel, optionally two time steps per launch.
//
// Same update as fwd_step_kernel (k_stencil.cu), i.e. compute_pressure +
// compute_seismogram of src/modeling/modeling.cu:301-353 in Jacobi order:
//     Q^{t+1} = d * (v^2 dt^2/dh^2 * L(Q^t) + 2 Q^t - d * Q^{t-1}) + s_{t+1}
// with the receivers recording d * Q^t.
//
// Structure (B200): persistent CTAs walk a list of 128-row x TX-column tiles
// of all shots of the batch.  A producer warp issues cp.async.bulk.tensor
// loads of the next STAGES tiles (Q^t with its halo, Q^{t-1} and v), each
// stage completing on a `full` mbarrier; eight consumer warps compute from
// shared memory and release a stage on its `empty` mbarrier, so the memory
// system always has whole tiles in flight and consumer warps never wait for
// one another in one-level launches.  With T = 2 the tile is loaded with an
// 8-cell halo, Q^{t+1} is computed on the tile plus a 4-cell ring in shared
// memory, and Q^{t+2} on the tile: every launch advances two time levels and
// writes both (out of place, into the other buffer pair), so a grid point
// costs 16 bytes of DRAM traffic per two updates instead of per update.
// Receivers are recorded from shared memory by the tile that owns them; the
// source is added by the writer of its point.  Waits are bounded: on a
// timeout the kernel raises *err and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include "kargs.h"
#include "kernels.h"
#include "fwd_tile.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace fwi {

namespace {

using namespace ft;

template <int T, int TX, int S, bool ABC>
__global__ void __launch_bounds__(kNT, 2)
    fwd_tma_kernel(const __grid_constant__ CUtensorMap m_cur, const __grid_constant__ CUtensorMap m_old,
                   const __grid_constant__ CUtensorMap m_vel, const FwdTmaArgs a) {
    using G = Geom<T, TX>;
    extern __shared__ __align__(128) float smem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t empty[S];
    __shared__ TileMeta meta[S];
    __shared__ int abort_flag;
    const int tid = threadIdx.x;
    const int total = __ldg(a.tile_base + a.ns);

    if (tid == 0) {
        for (int k = 0; k < S; ++k) {
            tma::mbar_init(&full[k], 1);
            tma::mbar_init(&empty[k], kNC / 32);
        }
        abort_flag = 0;
        tma::fence_barrier_init();
    }
    __syncthreads();

    if (tid >= kNC) {
        // ---------------- producer warp: one elected lane issues the loads
        if (tid != kNC) return;
        tma::prefetch_map(&m_cur);
        tma::prefetch_map(&m_old);
        tma::prefetch_map(&m_vel);
        int k = 0;
        for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++k) {
            const int stg = k % S;
            if (k >= S && !tma::mbar_wait(&empty[stg], (uint32_t)(((k / S) - 1) & 1), a.spin)) {
                atomicExch(a.err, 1);
                break;
            }
            const TileInfo ti = decode(a, tile, TX);
            const ShotDesc sd = a.shots[ti.s];
            TileMeta& mt = meta[stg];
            mt.s = ti.s;
            mt.x0 = ti.x0;
            mt.z0 = ti.z0;
            mt.nxx = sd.nxx;
            mt.col_off = sd.col_off;
            mt.has_src = (a.sample1 >= 0 || (T == 2 && a.sample2 >= 0)) &&
                         st::has_points(a.inj, sd.col_off, max(ti.x0 - 4, 0), min(ti.x0 + TX + 4, sd.nxx));
            if ((a.rec_sample0 >= 0 || a.rec_sample1 >= 0) && a.seis) {
                mt.rec_kb = __ldg(a.rec.colptr + sd.col_off + ti.x0);
                mt.rec_ke = __ldg(a.rec.colptr + sd.col_off + min(ti.x0 + TX, sd.nxx));
            } else {
                mt.rec_kb = mt.rec_ke = 0;
            }
            float* base = smem + stg * G::STAGE;
            // the arrive releases the meta writes to the consumers' acquiring wait
            tma::mbar_arrive_expect_tx(&full[stg], G::BYTES);
            tma::load_3d(base, &m_cur, ti.z0 - G::H, ti.x0 - G::H, ti.s, &full[stg]);
            tma::load_3d(base + G::CUR, &m_old, ti.z0 - (G::H - 4), ti.x0 - (G::H - 4), ti.s, &full[stg]);
            tma::load_3d(base + G::CUR + G::PTW, &m_vel, ti.z0 - (G::H - 4), ti.x0 - (G::H - 4) + sd.vel_col,
                         a.vel_shared ? 0 : ti.s, &full[stg]);
        }
        // never leave copies in flight behind an exiting CTA: wait (bounded)
        // for the last S loads issued
        for (int kk = (k > S ? k - S : 0); kk < k; ++kk) tma::mbar_wait(&full[kk % S], (uint32_t)((kk / S) & 1), a.spin);
        return;
    }

    // -------------------- consumer warps
    const int lane = tid & 31;
    int k = 0;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++k) {
        const int stg = k % S;
        bool ok = tma::mbar_wait(&full[stg], (uint32_t)((k / S) & 1), a.spin);
        if (T == 2) {
            // the ring tile is shared by all consumer warps: agree on going on
            if (!ok) abort_flag = 1;
            consumer_barrier();
            ok = abort_flag == 0;
        }
        if (!ok) {
            if (lane == 0) atomicExch(a.err, 1);
            break;
        }
        const TileMeta mt = meta[stg];
        Tile t;
        t.ti.s = mt.s;
        t.ti.x0 = mt.x0;
        t.ti.z0 = mt.z0;
        t.nxx = mt.nxx;
        t.col_off = mt.col_off;
        t.cur = smem + stg * G::STAGE;
        t.old = t.cur + G::CUR;
        t.vel = t.old + G::PTW;
        t.mid = smem + S * G::STAGE;
        t.has_src = mt.has_src != 0;
        const float* b1d = ABC ? a.b1d : nullptr;

        if (T == 2) {
            const bool inner = st::tile_inner(t.ti.z0 - 4, kTZ + 8, t.ti.x0 - 4, TX + 8, a.nzz, t.nxx);
            const bool undamped = st::tile_undamped(b1d, a.nb, t.ti.z0 - 4, kTZ + 8, t.ti.x0 - 4, TX + 8, a.nzz, t.nxx);
            if (inner && undamped) mid_pass<T, TX, false, false>(a, t);
            else if (inner) mid_pass<T, TX, ABC, false>(a, t);
            else mid_pass<T, TX, ABC, true>(a, t);
            consumer_barrier();
        }

        // receivers owned by this tile: Q^t (and Q^{t+1}) from shared memory
        if (mt.rec_kb < mt.rec_ke) {
            const int xe = min(t.ti.x0 + TX, t.nxx);
            for (int r = mt.rec_kb + tid; r < mt.rec_ke; r += kNC) {
                const int z = __ldg(a.rec.z + r);
                if (z < t.ti.z0 || z >= t.ti.z0 + kTZ) continue;
                // column of the receiver: the last column whose colptr start is <= r
                int lo = t.ti.x0, hi = xe;
                while (hi - lo > 1) {
                    const int m = (lo + hi) >> 1;
                    if (__ldg(a.rec.colptr + t.col_off + m) <= r) lo = m;
                    else hi = m;
                }
                const int x = lo;
                const float d = ABC ? st::damp(st::rows_info(a.b1d, a.nb, z, a.nzz),
                                               st::col_info(a.b1d, a.nb, x, t.nxx), 0)
                                    : 1.0f;
                const long long so = __ldg(a.rec.soff + r);
                if (a.rec_sample0 >= 0)
                    a.seis[so + a.rec_sample0] = d * t.cur[(x - t.ti.x0 + G::H) * G::CZ + (z - t.ti.z0 + G::H)];
                if (T == 2 && a.rec_sample1 >= 0)
                    a.seis[so + a.rec_sample1] = d * t.mid[(x - t.ti.x0 + 4) * G::MZ + (z - t.ti.z0 + 4)];
            }
        }

        {
            const bool inner = st::tile_inner(t.ti.z0, kTZ, t.ti.x0, TX, a.nzz, t.nxx);
            const bool undamped = st::tile_undamped(b1d, a.nb, t.ti.z0, kTZ, t.ti.x0, TX, a.nzz, t.nxx);
            if (inner && undamped) final_pass<T, TX, false, false>(a, t);
            else if (inner) final_pass<T, TX, ABC, false>(a, t);
            else final_pass<T, TX, ABC, true>(a, t);
        }
        __syncwarp();
        if (lane == 0) tma::mbar_arrive(&empty[stg]);  // this warp is done with stage `stg`
        if (T == 2) consumer_barrier();                // the ring tile is free again
    }
}

template <int T, int TX, int S>
constexpr size_t smem_bytes() {
    return (size_t)(S * Geom<T, TX>::STAGE + Geom<T, TX>::MID) * sizeof(float);
}

template <int T, int TX, int S, bool ABC>
cudaError_t configure_one(int* ctas) {
    auto fn = fwd_tma_kernel<T, TX, S, ABC>;
    const size_t smem = smem_bytes<T, TX, S>();
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, kNT, smem);
}

template <int T, int TX, int S>
cudaError_t configure_pair(int* ctas) {
    int a = 0, b = 0;
    cudaError_t e = configure_one<T, TX, S, true>(&a);
    if (e == cudaSuccess) e = configure_one<T, TX, S, false>(&b);
    *ctas = a < b ? a : b;
    return e;
}

template <int T, int TX, int S>
cudaError_t launch_variant(const CUtensorMap& mc, const CUtensorMap& mo, const CUtensorMap& mv, const FwdTmaArgs& a,
                           int grid, cudaStream_t st) {
    const size_t smem = smem_bytes<T, TX, S>();
    if (a.b1d) fwd_tma_kernel<T, TX, S, true><<<grid, kNT, smem, st>>>(mc, mo, mv, a);
    else fwd_tma_kernel<T, TX, S, false><<<grid, kNT, smem, st>>>(mc, mo, mv, a);
    return cudaGetLastError();
}

// The variants compiled: (T, TX, S).
#define FWI_FWD_TMA_VARIANTS(X) X(1, 32, 2) X(1, 32, 3) X(1, 16, 3) X(1, 16, 4) X(2, 32, 2) X(2, 16, 2) X(2, 16, 3)

}  // namespace

int fwd_tma_rows() { return kTZ; }

bool fwd_tma_supported(const FwdTmaConfig& c) {
#define FWI_X(t, tx, s) if (c.T == t && c.TX == tx && c.S == s) return true;
    FWI_FWD_TMA_VARIANTS(FWI_X)
#undef FWI_X
    return false;
}

size_t fwd_tma_smem(const FwdTmaConfig& c) {
#define FWI_X(t, tx, s) if (c.T == t && c.TX == tx && c.S == s) return smem_bytes<t, tx, s>();
    FWI_FWD_TMA_VARIANTS(FWI_X)
#undef FWI_X
    return 0;
}

int fwd_tma_box_cur_z(const FwdTmaConfig& c) { return kTZ + 8 * c.T; }
int fwd_tma_box_cur_x(const FwdTmaConfig& c) { return c.TX + 8 * c.T; }
int fwd_tma_box_pt_z(const FwdTmaConfig& c) { return kTZ + 8 * (c.T - 1); }
int fwd_tma_box_pt_x(const FwdTmaConfig& c) { return c.TX + 8 * (c.T - 1); }

cudaError_t fwd_tma_configure(int* ctas_per_sm, const FwdTmaConfig& c) {
#define FWI_X(t, tx, s) if (c.T == t && c.TX == tx && c.S == s) return configure_pair<t, tx, s>(ctas_per_sm);
    FWI_FWD_TMA_VARIANTS(FWI_X)
#undef FWI_X
    return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_tma(const FwdTmaConfig& c, const CUtensorMap& m_cur, const CUtensorMap& m_old,
                           const CUtensorMap& m_vel, const FwdTmaArgs& a, int grid, cudaStream_t st) {
#define FWI_X(t, tx, s) \
    if (c.T == t && c.TX == tx && c.S == s) return launch_variant<t, tx, s>(m_cur, m_old, m_vel, a, grid, st);
    FWI_FWD_TMA_VARIANTS(FWI_X)
#undef FWI_X
    return cudaErrorInvalidValue;
}

}  // namespace fwi
