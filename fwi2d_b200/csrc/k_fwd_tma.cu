// k_fwd_tma.cu — forward leapfrog steps with TMA-staged tiles in a persistent,
// pipelined kernel, optionally two time steps per launch.
//
// Same update as fwd_step_kernel (k_stencil.cu), i.e. compute_pressure +
// compute_seismogram of src/modeling/modeling.cu:301-353 in Jacobi order:
//     Q^{t+1} = d * (v^2 dt^2/dh^2 * L(Q^t) + 2 Q^t - d * Q^{t-1}) + s_{t+1}
// with the receivers recording d * Q^t.
//
// Structure (B200): one CTA per SM walks a list of 128-row x TX-column tiles
// of all shots of the batch.  Thread 0 issues cp.async.bulk.tensor loads of
// the next STAGES tiles (Q^t with its halo, Q^{t-1} and v) onto an mbarrier per
// stage, so the memory system always has whole tiles in flight while the
// CTA computes from shared memory.  With T = 2 the tile is loaded with an
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
#include "tma.cuh"

namespace fwi {

namespace {

constexpr int kTZ = 128;   // output rows per tile
constexpr int kNT = 256;   // threads per CTA

template <int T, int TX>
struct Geom {
    static constexpr int H = 4 * T;                 // halo of the Q^t tile
    static constexpr int CZ = kTZ + 2 * H;          // rows of the Q^t tile
    static constexpr int CX = TX + 2 * H;           // columns of the Q^t tile
    static constexpr int PZ = kTZ + 2 * (H - 4);    // rows of the Q^{t-1} and v tiles
    static constexpr int PX = TX + 2 * (H - 4);
    static constexpr int CUR = CZ * CX;
    static constexpr int PTW = PZ * PX;
    static constexpr int STAGE = CUR + 2 * PTW;     // floats per pipeline stage
    static constexpr int MZ = kTZ + 8, MX = TX + 8; // Q^{t+1} ring tile (T = 2)
    static constexpr int MID = (T == 2) ? MZ * MX : 0;
    static constexpr uint32_t BYTES = STAGE * 4;
    static_assert((CUR * 4) % 128 == 0 && (PTW * 4) % 128 == 0, "TMA destinations must stay 128-byte aligned");
    static_assert(CZ <= 256 && CX <= 256, "TMA box extent");
};

__device__ __forceinline__ float el(const float4& v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

// dh^2 * Laplacian at rows r..r+3 (r % 4 == 0) of column c of a shared tile
// whose columns hold LD floats.
template <int LD>
__device__ __forceinline__ void lap4(const float* t, int r, int c, float out[4]) {
    const float c0 = (float)(-2.0 * kFDM5), c1 = (float)kFDM4, c2 = (float)(-kFDM3), c3 = (float)kFDM2,
                c4 = (float)(-kFDM1);
    const float* col = t + c * LD + r;
    const float4 up = *reinterpret_cast<const float4*>(col - 4);
    const float4 own = *reinterpret_cast<const float4*>(col);
    const float4 dn = *reinterpret_cast<const float4*>(col + 4);
    const float z[12] = {up.x, up.y, up.z, up.w, own.x, own.y, own.z, own.w, dn.x, dn.y, dn.z, dn.w};
    float4 xm[4], xp[4];
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        xm[k - 1] = *reinterpret_cast<const float4*>(col - k * LD);
        xp[k - 1] = *reinterpret_cast<const float4*>(col + k * LD);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float s1 = (el(xm[0], e) + el(xp[0], e)) + (z[e + 3] + z[e + 5]);
        const float s2 = (el(xm[1], e) + el(xp[1], e)) + (z[e + 2] + z[e + 6]);
        const float s3 = (el(xm[2], e) + el(xp[2], e)) + (z[e + 1] + z[e + 7]);
        const float s4 = (el(xm[3], e) + el(xp[3], e)) + (z[e + 0] + z[e + 8]);
        float l = c4 * s4;
        l = fmaf(c3, s3, l);
        l = fmaf(c2, s2, l);
        l = fmaf(c1, s1, l);
        out[e] = fmaf(c0, z[e + 4], l);
    }
}

// Cerjan damper in closed form (see k_stencil.cu); i, j inside the grid.
__device__ __forceinline__ float damper(const float* __restrict__ b1d, int nb, int i, int j, int nzz, int nxx) {
    const int iz = i < nb ? i : (i >= nzz - nb ? nzz - 1 - i : -1);
    const int jx = j < nb ? j : (j >= nxx - nb ? nxx - 1 - j : -1);
    const float dz = iz >= 0 ? __ldg(b1d + iz) : 1.0f;
    const float dx = jx >= 0 ? __ldg(b1d + jx) : 1.0f;
    return (iz >= 0 && jx >= 0) ? (dz + dx) - 1.0f : dz * dx;
}

// Source amplitude added at rows z..z+3 of column j (j inside the grid).
__device__ __forceinline__ void inject4(const InjTable& inj, int sample, int col_off, int j, int z, float v[4]) {
    if (sample < 0) return;
    const int kb = __ldg(inj.colptr + col_off + j), ke = __ldg(inj.colptr + col_off + j + 1);
    for (int k = kb; k < ke; ++k) {
        const int dz = __ldg(inj.z + k) - z;
        if (dz >= 0 && dz < 4) {
            const float amp = inj.scale * __ldg(inj.series + __ldg(inj.soff + k) + sample);
            if (dz == 0) v[0] += amp;
            else if (dz == 1) v[1] += amp;
            else if (dz == 2) v[2] += amp;
            else v[3] += amp;
        }
    }
}

struct TileInfo {
    int s, x0, z0;
};

__device__ __forceinline__ TileInfo decode(const FwdTmaArgs& a, int tile, int tx_width) {
    int lo = 0, hi = a.ns;  // tile_base[lo] <= tile < tile_base[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(a.tile_base + mid) <= tile) lo = mid;
        else hi = mid;
    }
    const int local = tile - __ldg(a.tile_base + lo);
    TileInfo ti;
    ti.s = lo;
    ti.z0 = (local % a.ntz) * kTZ;
    ti.x0 = (local / a.ntz) * tx_width;
    return ti;
}

template <int T, int TX, int S, bool ABC>
__global__ void __launch_bounds__(kNT, 2)
    fwd_tma_kernel(const __grid_constant__ CUtensorMap m_cur, const __grid_constant__ CUtensorMap m_old,
                   const __grid_constant__ CUtensorMap m_vel, const FwdTmaArgs a) {
    using G = Geom<T, TX>;
    extern __shared__ __align__(128) float smem[];
    __shared__ __align__(8) uint64_t full[S];
    float* mid = smem + S * G::STAGE;
    const int tid = threadIdx.x;
    const int total = __ldg(a.tile_base + a.ns);

    if (tid == 0) {
        tma::prefetch_map(&m_cur);
        tma::prefetch_map(&m_old);
        tma::prefetch_map(&m_vel);
        for (int k = 0; k < S; ++k) tma::mbar_init(&full[k], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int tile, int st) {
        const TileInfo ti = decode(a, tile, TX);
        float* base = smem + st * G::STAGE;
        tma::mbar_arrive_expect_tx(&full[st], G::BYTES);
        tma::load_3d(base, &m_cur, ti.z0 - G::H, ti.x0 - G::H, ti.s, &full[st]);
        tma::load_3d(base + G::CUR, &m_old, ti.z0 - (G::H - 4), ti.x0 - (G::H - 4), ti.s, &full[st]);
        tma::load_3d(base + G::CUR + G::PTW, &m_vel, ti.z0 - (G::H - 4), ti.x0 - (G::H - 4),
                     a.vel_shared ? 0 : ti.s, &full[st]);
    };

    int issued = 0;  // tiles issued by this CTA
    if (tid == 0)
        for (int k = 0; k < S; ++k) {
            const int tile = blockIdx.x + k * gridDim.x;
            if (tile < total) {
                issue(tile, k);
                ++issued;
            }
        }

    const int lane = tid & 31, warp = tid >> 5;
    const float k2 = a.dt2idh2;
    int k = 0;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++k) {
        const int st = k % S;
        const bool ok = tma::mbar_wait(&full[st], (uint32_t)((k / S) & 1));
        if (!__syncthreads_and(ok)) {
            if (tid == 0) atomicExch(a.err, 1);
            break;
        }
        const TileInfo ti = decode(a, tile, TX);
        const ShotDesc sd = a.shots[ti.s];
        const int nxx = sd.nxx;
        const float* cur = smem + st * G::STAGE;
        const float* old = cur + G::CUR;
        const float* vel = old + G::PTW;

        if (T == 2) {
            // Q^{t+1} on the tile and a 4-cell ring around it
            constexpr int QZ = G::MZ / 4;
            for (int w = tid; w < QZ * G::MX; w += kNT) {
                const int q = w % QZ, c = w / QZ;
                const int gx = ti.x0 - 4 + c, gz = ti.z0 - 4 + 4 * q;
                float out[4] = {0.f, 0.f, 0.f, 0.f};
                if (gx >= 4 && gx < nxx - 4) {
                    float l[4];
                    lap4<G::CZ>(cur, 4 * q + 4, c + 4, l);
                    const float4 qq = *reinterpret_cast<const float4*>(cur + (c + 4) * G::CZ + 4 * q + 4);
                    const float4 oo = *reinterpret_cast<const float4*>(old + c * G::PZ + 4 * q);
                    const float4 vv = *reinterpret_cast<const float4*>(vel + c * G::PZ + 4 * q);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int i = gz + e;
                        if (i >= 4 && i < a.nzz - 4) {
                            const float v = el(vv, e);
                            const float kk = k2 * (v * v);
                            if (ABC) {
                                const float d = damper(a.b1d, a.nb, i, gx, a.nzz, nxx);
                                out[e] = d * (kk * l[e] + 2.0f * el(qq, e) - d * el(oo, e));
                            } else {
                                out[e] = kk * l[e] + 2.0f * el(qq, e) - el(oo, e);
                            }
                        }
                    }
                }
                if (gx >= 0 && gx < nxx) inject4(a.inj, a.sample1, sd.col_off, gx, gz, out);
                *reinterpret_cast<float4*>(mid + c * G::MZ + 4 * q) = make_float4(out[0], out[1], out[2], out[3]);
            }
            __syncthreads();
        }

        // receivers owned by this tile: Q^t (and Q^{t+1}) from shared memory
        if ((a.rec_sample0 >= 0 || a.rec_sample1 >= 0) && a.seis) {
            const int xe = min(ti.x0 + TX, nxx);
            const int kb = __ldg(a.rec.colptr + sd.col_off + ti.x0), ke = __ldg(a.rec.colptr + sd.col_off + xe);
            for (int r = kb + tid; r < ke; r += kNT) {
                const int z = __ldg(a.rec.z + r);
                if (z < ti.z0 || z >= ti.z0 + kTZ) continue;
                // column of the receiver: the last column whose colptr start is <= r
                int lo = ti.x0, hi = xe;
                while (hi - lo > 1) {
                    const int m = (lo + hi) >> 1;
                    if (__ldg(a.rec.colptr + sd.col_off + m) <= r) lo = m;
                    else hi = m;
                }
                const int x = lo;
                const float d = ABC ? damper(a.b1d, a.nb, z, x, a.nzz, nxx) : 1.0f;
                const long long so = __ldg(a.rec.soff + r);
                if (a.rec_sample0 >= 0)
                    a.seis[so + a.rec_sample0] = d * cur[(x - ti.x0 + G::H) * G::CZ + (z - ti.z0 + G::H)];
                if (T == 2 && a.rec_sample1 >= 0)
                    a.seis[so + a.rec_sample1] = d * mid[(x - ti.x0 + 4) * G::MZ + (z - ti.z0 + 4)];
            }
        }

        // last level of the launch on the tile
        {
            const int p = lane;
            const int z = ti.z0 + 4 * p;
            constexpr int CPW = TX / 8;  // columns per warp
            if (z < a.ldz) {
#pragma unroll 1
                for (int j = 0; j < CPW; ++j) {
                    const int c = warp * CPW + j;
                    const int gx = ti.x0 + c;
                    if (gx >= nxx) break;
                    float out[4] = {0.f, 0.f, 0.f, 0.f};
                    const size_t goff = (size_t)ti.s * a.fstride + (size_t)gx * a.ldz + z;
                    if (T == 2) {
                        const float4 m1 = *reinterpret_cast<const float4*>(mid + (c + 4) * G::MZ + 4 * p + 4);
                        *reinterpret_cast<float4*>(a.out1 + goff) = m1;
                    }
                    if (gx >= 4 && gx < nxx - 4) {
                        float l[4];
                        float4 qq, oo;
                        if (T == 2) {
                            lap4<G::MZ>(mid, 4 * p + 4, c + 4, l);
                            qq = *reinterpret_cast<const float4*>(mid + (c + 4) * G::MZ + 4 * p + 4);
                            oo = *reinterpret_cast<const float4*>(cur + (c + 8) * G::CZ + 4 * p + 8);
                        } else {
                            lap4<G::CZ>(cur, 4 * p + 4, c + 4, l);
                            qq = *reinterpret_cast<const float4*>(cur + (c + 4) * G::CZ + 4 * p + 4);
                            oo = *reinterpret_cast<const float4*>(old + c * G::PZ + 4 * p);
                        }
                        const float4 vv = *reinterpret_cast<const float4*>(vel + (c + G::H - 4) * G::PZ + 4 * p +
                                                                             (G::H - 4));
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const int i = z + e;
                            if (i >= 4 && i < a.nzz - 4) {
                                const float v = el(vv, e);
                                const float kk = k2 * (v * v);
                                if (ABC) {
                                    const float d = damper(a.b1d, a.nb, i, gx, a.nzz, nxx);
                                    out[e] = d * (kk * l[e] + 2.0f * el(qq, e) - d * el(oo, e));
                                } else {
                                    out[e] = kk * l[e] + 2.0f * el(qq, e) - el(oo, e);
                                }
                            }
                        }
                    }
                    inject4(a.inj, T == 2 ? a.sample2 : a.sample1, sd.col_off, gx, z, out);
                    float* dst = (T == 2 ? a.out2 : a.out1) + goff;
                    *reinterpret_cast<float4*>(dst) = make_float4(out[0], out[1], out[2], out[3]);
                }
            }
        }
        __syncthreads();  // stage `st` (and the ring tile) are free again
        if (tid == 0) {
            const int next = tile + S * gridDim.x;
            if (next < total) {
                issue(next, st);
                ++issued;
            }
        }
    }
    // a timed-out CTA still owns its in-flight copies: wait for them (bounded)
    if (tid == 0 && k < issued) {
        for (int kk = k; kk < issued; ++kk) tma::mbar_wait(&full[kk % S], (uint32_t)((kk / S) & 1));
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
