// k_stencil.cu — one leapfrog time step of the 8th-order acoustic stencil for
// every shot of a batch in one launch.
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
// are staged in shared memory with a 4-cell halo (float4 rows along z, the
// contiguous axis).  Each thread produces a float4 (4 rows) in 4 columns.
#include <cuda_runtime.h>

#include "kargs.h"
#include "kernels.h"

namespace fwi {

namespace {

constexpr int kTZ4 = 32;                 // float4 rows per tile -> 128 rows
constexpr int kTX = 32;                  // columns per tile
constexpr int kH = 4;                    // stencil radius
constexpr int kSW = kTZ4 + 2;            // float4 rows incl. halo
constexpr int kSC = kTX + 2 * kH;        // columns incl. halo
constexpr int kThreads = 256;            // 32 lanes (z) x 8 (x)

__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }

__device__ __forceinline__ float get(const float4& v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

// Stage columns x0-4 .. x0+35, rows z0-4 .. z0+131 of field f (zeros outside).
__device__ __forceinline__ void load_tile(float4 (*t)[kSW], const float* __restrict__ f, int ldz, int nxx,
                                          int z0, int x0) {
    const int tid = threadIdx.x + threadIdx.y * 32;
    for (int idx = tid; idx < kSC * kSW; idx += kThreads) {
        const int c = idx / kSW, q = idx - c * kSW;
        const int gx = x0 - kH + c, gz = z0 - 4 + 4 * q;
        float4 v = zero4();
        if (gx >= 0 && gx < nxx && gz >= 0 && gz < ldz)
            v = __ldg(reinterpret_cast<const float4*>(f + (size_t)gx * ldz + gz));
        t[c][q] = v;
    }
}

// Laplacian times dh^2 at the 4 rows of thread `lane` in smem column c.
__device__ __forceinline__ void laplacian4(const float4 (*t)[kSW], int c, int lane, float lap[4]) {
    const float c0 = (float)(-2.0 * kFDM5), c1 = (float)kFDM4, c2 = (float)(-kFDM3), c3 = (float)kFDM2,
                c4 = (float)(-kFDM1);
    const float4 up = t[c][lane], own = t[c][lane + 1], dn = t[c][lane + 2];
    const float col[12] = {up.x, up.y, up.z, up.w, own.x, own.y, own.z, own.w, dn.x, dn.y, dn.z, dn.w};
    float4 xm[4], xp[4];
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        xm[k - 1] = t[c - k][lane + 1];
        xp[k - 1] = t[c + k][lane + 1];
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float s1 = (get(xm[0], e) + get(xp[0], e)) + (col[e + 3] + col[e + 5]);
        const float s2 = (get(xm[1], e) + get(xp[1], e)) + (col[e + 2] + col[e + 6]);
        const float s3 = (get(xm[2], e) + get(xp[2], e)) + (col[e + 1] + col[e + 7]);
        const float s4 = (get(xm[3], e) + get(xp[3], e)) + (col[e + 0] + col[e + 8]);
        float l = c4 * s4;
        l = fmaf(c3, s3, l);
        l = fmaf(c2, s2, l);
        l = fmaf(c1, s1, l);
        lap[e] = fmaf(c0, col[e + 4], l);
    }
}

// Cerjan damper of the reference's 9-region lookup (modeling.cu:355-402) in
// closed form: 1-D profiles dz(i), dx(j); inside a corner b2d = (dz+dx)-1,
// elsewhere the one profile that is not 1.
__device__ __forceinline__ float damper(const float* __restrict__ b1d, int nb, int i, int j, int nzz, int nxx) {
    const int iz = i < nb ? i : (i >= nzz - nb ? nzz - 1 - i : -1);
    const int jx = j < nb ? j : (j >= nxx - nb ? nxx - 1 - j : -1);
    const float dz = iz >= 0 ? __ldg(b1d + iz) : 1.0f;
    const float dx = jx >= 0 ? __ldg(b1d + jx) : 1.0f;
    return (iz >= 0 && jx >= 0) ? (dz + dx) - 1.0f : dz * dx;
}

// Injections of column j of a shot into the 4 rows z..z+3.
__device__ __forceinline__ void inject4(const InjTable& inj, int col_off, int j, int z, float v[4]) {
    if (inj.sample < 0) return;
    const int kb = __ldg(inj.colptr + col_off + j), ke = __ldg(inj.colptr + col_off + j + 1);
    for (int k = kb; k < ke; ++k) {
        const int dz = __ldg(inj.z + k) - z;
        if (dz >= 0 && dz < 4) {
            const float a = inj.scale * __ldg(inj.series + __ldg(inj.soff + k) + inj.sample);
            if (dz == 0) v[0] += a;
            else if (dz == 1) v[1] += a;
            else if (dz == 2) v[2] += a;
            else v[3] += a;
        }
    }
}

template <bool kABC>
__global__ void __launch_bounds__(kThreads) fwd_step_kernel(FwdArgs a) {
    __shared__ float4 tile[kSC][kSW];
    const int s = blockIdx.z;
    const ShotDesc sd = a.shots[s];
    const int nxx = sd.nxx;
    const int z0 = blockIdx.x * (4 * kTZ4), x0 = blockIdx.y * kTX;
    const float* cur = a.cur + (size_t)s * a.fstride;
    float* nxt = a.nxt + (size_t)s * a.fstride;
    const float* vel = a.vel + (size_t)s * a.vel_stride;

    // Receivers read Q^t, which this launch never writes.
    if (a.rec_sample >= 0 && blockIdx.x == 0 && blockIdx.y == 0) {
        for (int r = threadIdx.x + threadIdx.y * 32; r < sd.nrec; r += kThreads) {
            const int pt = __ldg(a.rec_pt + sd.rec_off + r);
            float v = __ldg(cur + pt);
            if (kABC) v *= damper(a.b1d, a.nb, pt % a.ldz, pt / a.ldz, a.nzz, nxx);
            a.seis[sd.seis_off + (long long)r * a.nt + a.rec_sample] = v;
        }
    }
    if (x0 >= nxx) return;

    load_tile(tile, cur, a.ldz, nxx, z0, x0);
    __syncthreads();

    const int lane = threadIdx.x, ty = threadIdx.y;
    const int z = z0 + 4 * lane;
    if (z >= a.ldz) return;
#pragma unroll 1
    for (int m = 0; m < 4; ++m) {
        const int lc = 4 * ty + m;
        const int j = x0 + lc;
        if (j >= nxx) break;
        float lap[4];
        laplacian4(tile, lc + kH, lane, lap);
        const float4 q = tile[lc + kH][lane + 1];
        const size_t off = (size_t)j * a.ldz + z;
        const float4 vv = __ldg(reinterpret_cast<const float4*>(vel + off));
        const float4 old = *reinterpret_cast<const float4*>(nxt + off);
        float out[4];
        const bool colok = (j >= 4) && (j < nxx - 4);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int i = z + e;
            const float v = get(vv, e);
            const float k = a.dt2idh2 * (v * v);
            float o = get(old, e), qq = get(q, e);
            float r;
            if (kABC) {
                const float d = damper(a.b1d, a.nb, i, j, a.nzz, nxx);
                r = d * (k * lap[e] + 2.0f * qq - d * o);
            } else {
                r = k * lap[e] + 2.0f * qq - o;
            }
            out[e] = (colok && i >= 4 && i < a.nzz - 4) ? r : 0.0f;
        }
        inject4(a.inj, sd.col_off, j, z, out);
        *reinterpret_cast<float4*>(nxt + off) = make_float4(out[0], out[1], out[2], out[3]);
    }
}

template <bool kGrad>
__global__ void __launch_bounds__(kThreads) bwd_step_kernel(BwdArgs a) {
    __shared__ float4 ts[kSC][kSW];
    __shared__ float4 tr[kSC][kSW];
    const int s = blockIdx.z;
    const ShotDesc sd = a.shots[s];
    const int nxx = sd.nxx;
    const int z0 = blockIdx.x * (4 * kTZ4), x0 = blockIdx.y * kTX;
    if (x0 >= nxx) return;
    const size_t fo = (size_t)s * a.fstride;
    const float* vel = a.vel + (size_t)s * a.vel_stride;
    float* acc_a = a.acc_a + (size_t)s * a.acc_stride;
    float* acc_b = a.acc_b + (size_t)s * a.acc_stride;

    load_tile(ts, a.ps_st + fo, a.ldz, nxx, z0, x0);
    load_tile(tr, a.pr_st + fo, a.ldz, nxx, z0, x0);
    __syncthreads();

    const int lane = threadIdx.x, ty = threadIdx.y;
    const int z = z0 + 4 * lane;
    if (z >= a.ldz) return;
#pragma unroll 1
    for (int m = 0; m < 4; ++m) {
        const int lc = 4 * ty + m;
        const int j = x0 + lc;
        if (j >= nxx) break;
        float ls[4], lr[4];
        laplacian4(ts, lc + kH, lane, ls);
        laplacian4(tr, lc + kH, lane, lr);
        const float4 psold = ts[lc + kH][lane + 1];
        const float4 pr = tr[lc + kH][lane + 1];
        const size_t off = (size_t)j * a.ldz + z;
        const float4 vv = __ldg(reinterpret_cast<const float4*>(vel + off));
        const float4 ps = *reinterpret_cast<const float4*>(a.ps_io + fo + off);
        const float4 prold = *reinterpret_cast<const float4*>(a.pr_io + fo + off);
        float4 ga = *reinterpret_cast<const float4*>(acc_a + off);
        float4 gb = *reinterpret_cast<const float4*>(acc_b + off);
        float nps[4], npr[4], na[4], nb4[4];
        const bool colok = (j >= 4) && (j < nxx - 4);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int i = z + e;
            const bool ok = colok && i >= 4 && i < a.nzz - 4;
            const float v = get(vv, e);
            const float vp2 = v * v;
            const float k = a.dt2idh2 * vp2;
            const float s_new = k * ls[e] + 2.0f * get(psold, e) - get(ps, e);
            const float r_new = k * lr[e] + 2.0f * get(pr, e) - get(prold, e);
            nps[e] = ok ? s_new : 0.0f;
            npr[e] = ok ? r_new : 0.0f;
            const float prv = get(pr, e);
            float da, db;
            if (kGrad) da = a.dt * prv * (ls[e] * a.idh2) * vp2;
            else da = s_new * prv;
            db = s_new * s_new;
            na[e] = get(ga, e) + (ok ? da : 0.0f);
            nb4[e] = get(gb, e) + (ok ? db : 0.0f);
        }
        inject4(a.inj, sd.col_off, j, z, npr);
        *reinterpret_cast<float4*>(a.ps_io + fo + off) = make_float4(nps[0], nps[1], nps[2], nps[3]);
        *reinterpret_cast<float4*>(a.pr_io + fo + off) = make_float4(npr[0], npr[1], npr[2], npr[3]);
        *reinterpret_cast<float4*>(acc_a + off) = make_float4(na[0], na[1], na[2], na[3]);
        *reinterpret_cast<float4*>(acc_b + off) = make_float4(nb4[0], nb4[1], nb4[2], nb4[3]);
    }
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
