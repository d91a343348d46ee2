// k_stencil.cu — one leapfrog time step of the 8th-order acoustic stencil for
// every shot of a batch in one launch (shared-memory tiles, one tile per CTA).
//
// Forward step (replaces compute_pressure + compute_seismogram,
// src/modeling/modeling.cu:301-353).  The buffers hold the field *after* the
// source injection of its time level, Q^t = p^t + s_t at the source, so one
// launch reads Q^t through the stencil and Q^{t-1} pointwise and writes
//     Q^{t+1} = d * (v^2 dt^2/dh^2 * L(Q^t) + 2 Q^t - d * Q^{t-1}) + s_{t+1}
// where d is the Cerjan damper of the reference (1 without ABC) and L the
// 8th-order Laplacian times dh^2.  This is the reference's update with its two
// in-place writes (P += s, P *= d) moved to the writer of each point, so all
// reads see the previous time level (Jacobi order) and no atomics are needed.
// Receivers record d * Q^t, the damped value compute_seismogram reads.
//
// Backward step (replaces inject_seismogram/inject_adjoint + cross_correlation
// / build_gradient, migration.cu:117-180, inversion.cu:381-444): the source
// field is stepped back in time and the receiver field forward, and the
// zero-lag image (Ps_new * Pr) or gradient (dt * Pr * v^2 * lap(Psold)) and the
// illumination (Ps_new^2) accumulate per shot.
//
// Tiling: a CTA owns 128 rows x 32 columns of one shot; the stencil field(s)
// are staged in shared memory with a 4-cell halo.  A thread produces 4 rows
// (one float4 along z, the contiguous axis) in 4 consecutive columns, reading
// the 12 columns of its x stencil once (stencil.cuh).
#include <cuda_runtime.h>

#include "kargs.h"
#include "kernels.h"
#include "stencil.cuh"

namespace fwi {

namespace {

constexpr int kTZ4 = 32;                 // float4 rows per tile -> 128 rows
constexpr int kTX = 32;                  // columns per tile
constexpr int kH = 4;                    // stencil radius
constexpr int kSW = kTZ4 + 2;            // float4 rows incl. halo
constexpr int kSC = kTX + 2 * kH;        // columns incl. halo
constexpr int kLD = 4 * kSW;             // floats per smem column
constexpr int kThreads = 256;            // 32 lanes (z) x 8 (x)

// Stage columns x0-4 .. x0+35, rows z0-4 .. z0+131 of field f (zeros outside).
__device__ __forceinline__ void load_tile(float4 (*t)[kSW], const float* __restrict__ f, int ldz, int nxx,
                                          int z0, int x0) {
    for (int c = threadIdx.y; c < kSC; c += kThreads / 32) {
        const int gx = x0 - kH + c;
        const bool colok = gx >= 0 && gx < nxx;
        const float* src = f + (size_t)gx * ldz;
        for (int q = threadIdx.x; q < kSW; q += 32) {
            const int gz = z0 - 4 + 4 * q;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (colok && gz >= 0 && gz < ldz) v = __ldg(reinterpret_cast<const float4*>(src + gz));
            t[c][q] = v;
        }
    }
}

// Forward update of the 4 columns of thread (lane, ty) on a loaded tile, one
// column at a time (few live registers, so 3-4 CTAs share an SM).
template <bool DAMP, bool EDGE>
__device__ __forceinline__ void fwd_columns(const FwdArgs& a, const float* tilef, const ShotDesc& sd, int nxx,
                                            int x0, int z, const float* vel, float* nxt, bool has_src,
                                            const st::Rows& rows) {
    const int lane = threadIdx.x, ty = threadIdx.y;
#pragma unroll 1
    for (int m = 0; m < 4; ++m) {
        const int j = x0 + 4 * ty + m;
        if (j >= nxx) break;
        const size_t off = (size_t)j * a.ldz + z;
        const float4 vv = __ldg(reinterpret_cast<const float4*>(vel + off));
        const float4 old = *reinterpret_cast<const float4*>(nxt + off);
        float l[1][4];
        float4 q[1];
        st::lap_run<kLD, 1>(tilef, 4 * lane + 4, 4 * ty + kH + m, l, q);
        const st::Col col =
            (DAMP || EDGE) ? st::col_info(DAMP ? a.b1d : nullptr, a.nb, j, nxx) : st::Col{1.0f, false, true};
        float4 out = st::update4<DAMP, EDGE>(l[0], q[0], old, vv, a.dt2idh2, rows, col);
        if (has_src) st::inject4(a.inj, a.inj.sample, sd.col_off, j, z, out);
        *reinterpret_cast<float4*>(nxt + off) = out;
    }
}

template <bool kABC>
__global__ void __launch_bounds__(kThreads) fwd_step_kernel(FwdArgs a) {
    __shared__ __align__(16) float4 tile[kSC][kSW];
    const int s = blockIdx.z;
    const ShotDesc sd = a.shots[s];
    const int nxx = sd.nxx;
    const int z0 = blockIdx.x * (4 * kTZ4), x0 = blockIdx.y * kTX;
    const float* cur = a.cur + (size_t)s * a.fstride;
    float* nxt = a.nxt + (size_t)s * a.fstride;
    const float* vel = a.vel + (size_t)s * a.vel_stride + (size_t)sd.vel_col * a.ldz;

    // Receivers read Q^t, which this launch never writes.
    if (a.rec_sample >= 0 && blockIdx.x == 0 && blockIdx.y == 0) {
        for (int r = threadIdx.x + threadIdx.y * 32; r < sd.nrec; r += kThreads) {
            const int pt = __ldg(a.rec_pt + sd.rec_off + r);
            float v = __ldg(cur + pt);
            if (kABC) {
                const st::Rows rr = st::rows_info(a.b1d, a.nb, pt % a.ldz, a.nzz);
                v *= st::damp(rr, st::col_info(a.b1d, a.nb, pt / a.ldz, nxx), 0);
            }
            a.seis[__ldg(a.rec_soff + sd.rec_off + r) + a.rec_sample] = v;
        }
    }
    if (x0 >= nxx) return;

    const int z = z0 + 4 * threadIdx.x;
    const bool has_src = a.inj.sample >= 0 && st::has_points(a.inj, sd.col_off, x0, min(x0 + kTX, nxx));
    load_tile(tile, cur, a.ldz, nxx, z0, x0);
    __syncthreads();

    if (z >= a.ldz) return;
    const float* tilef = reinterpret_cast<const float*>(&tile[0][0]);
    const bool inner = st::tile_inner(z0, 4 * kTZ4, x0, kTX, a.nzz, nxx);
    const bool undamped = !kABC || st::tile_undamped(a.b1d, a.nb, z0, 4 * kTZ4, x0, kTX, a.nzz, nxx);
    const st::Rows rows = st::rows_info(kABC ? a.b1d : nullptr, a.nb, z, a.nzz);
    if (inner && undamped) fwd_columns<false, false>(a, tilef, sd, nxx, x0, z, vel, nxt, has_src, rows);
    else if (inner) fwd_columns<kABC, false>(a, tilef, sd, nxx, x0, z, vel, nxt, has_src, rows);
    else fwd_columns<kABC, true>(a, tilef, sd, nxx, x0, z, vel, nxt, has_src, rows);
}

template <bool kGrad, bool EDGE>
__device__ __forceinline__ void bwd_columns(const BwdArgs& a, const float* tsf, const float* trf, const ShotDesc& sd,
                                            int nxx, int x0, int z, size_t fo, const float* vel, float* acc_a,
                                            float* acc_b, bool has_rec, const st::Rows& rows) {
    const int lane = threadIdx.x, ty = threadIdx.y;
    float ls[4][4], lr[4][4];
    float4 psold[4], pr[4];
    st::lap_run<kLD, 4>(tsf, 4 * lane + 4, 4 * ty + kH, ls, psold);
    st::lap_run<kLD, 4>(trf, 4 * lane + 4, 4 * ty + kH, lr, pr);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int j = x0 + 4 * ty + m;
        if (j >= nxx) break;
        const size_t off = (size_t)j * a.ldz + z;
        const float4 vv = __ldg(reinterpret_cast<const float4*>(vel + off));
        const float4 ps = *reinterpret_cast<const float4*>(a.ps_io + fo + off);
        const float4 prold = *reinterpret_cast<const float4*>(a.pr_io + fo + off);
        const float4 ga = *reinterpret_cast<const float4*>(acc_a + off);
        const float4 gb = *reinterpret_cast<const float4*>(acc_b + off);
        const bool colok = !EDGE || (j >= 4 && j < nxx - 4);
        const st::Bwd4 r = st::bwd_update4<kGrad, EDGE>(ls[m], psold[m], lr[m], pr[m], ps, prold, vv, ga, gb,
                                                        a.dt2idh2, a.dt, a.idh2, rows, colok);
        float4 rv = r.pr;
        if (has_rec) st::inject4(a.inj, a.inj.sample, sd.col_off, j, z, rv);
        *reinterpret_cast<float4*>(a.ps_io + fo + off) = r.ps;
        *reinterpret_cast<float4*>(a.pr_io + fo + off) = rv;
        *reinterpret_cast<float4*>(acc_a + off) = r.a;
        *reinterpret_cast<float4*>(acc_b + off) = r.b;
    }
}

template <bool kGrad>
__global__ void __launch_bounds__(kThreads) bwd_step_kernel(BwdArgs a) {
    __shared__ __align__(16) float4 ts[kSC][kSW];
    __shared__ __align__(16) float4 tr[kSC][kSW];
    const int s = blockIdx.z;
    const ShotDesc sd = a.shots[s];
    const int nxx = sd.nxx;
    const int z0 = blockIdx.x * (4 * kTZ4), x0 = blockIdx.y * kTX;
    if (x0 >= nxx) return;
    const size_t fo = (size_t)s * a.fstride;
    const float* vel = a.vel + (size_t)s * a.vel_stride + (size_t)sd.vel_col * a.ldz;
    float* acc_a = a.acc_a + (size_t)s * a.acc_stride;
    float* acc_b = a.acc_b + (size_t)s * a.acc_stride;

    load_tile(ts, a.ps_st + fo, a.ldz, nxx, z0, x0);
    load_tile(tr, a.pr_st + fo, a.ldz, nxx, z0, x0);
    __syncthreads();

    const int z = z0 + 4 * threadIdx.x;
    if (z >= a.ldz) return;
    const bool has_rec = a.inj.sample >= 0 && st::has_points(a.inj, sd.col_off, x0, min(x0 + kTX, nxx));
    const st::Rows rows = st::rows_info(nullptr, 0, z, a.nzz);
    const float* tsf = reinterpret_cast<const float*>(&ts[0][0]);
    const float* trf = reinterpret_cast<const float*>(&tr[0][0]);
    if (st::tile_inner(z0, 4 * kTZ4, x0, kTX, a.nzz, nxx))
        bwd_columns<kGrad, false>(a, tsf, trf, sd, nxx, x0, z, fo, vel, acc_a, acc_b, has_rec, rows);
    else
        bwd_columns<kGrad, true>(a, tsf, trf, sd, nxx, x0, z, fo, vel, acc_a, acc_b, has_rec, rows);
}

}  // namespace

dim3 step_grid(int ldz, int max_nxx, int nshots) {
    return dim3((unsigned)((ldz + 4 * kTZ4 - 1) / (4 * kTZ4)), (unsigned)((max_nxx + kTX - 1) / kTX),
                (unsigned)nshots);
}

void launch_fwd_step(const FwdArgs& a, dim3 grid, cudaStream_t st) {
    dim3 block(32, kThreads / 32);
    if (a.b1d) fwd_step_kernel<true><<<grid, block, 0, st>>>(a);
    else fwd_step_kernel<false><<<grid, block, 0, st>>>(a);
}

void launch_bwd_step(const BwdArgs& a, bool gradient, dim3 grid, cudaStream_t st) {
    dim3 block(32, kThreads / 32);
    if (gradient) bwd_step_kernel<true><<<grid, block, 0, st>>>(a);
    else bwd_step_kernel<false><<<grid, block, 0, st>>>(a);
}

}  // namespace fwi
