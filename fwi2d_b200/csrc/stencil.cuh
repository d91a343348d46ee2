// stencil.cuh — device helpers shared by the forward / backward step kernels.
//
// The update of every point is the reference's (compute_pressure,
// src/modeling/modeling.cu:301-345):
//     new = d * (v^2 dt^2/dh^2 * L + 2 q - d * old)        (d = 1 without ABC)
// zeroed outside 4 <= i < nzz-4, 4 <= j < nxx-4, with L = dh^2 * Laplacian from
// the 8th-order coefficients FDM1..5 (modeling.cuh:9-13).  The helpers below
// keep one operation order everywhere, so every kernel variant produces the
// same bits.  Tiles are classified once per CTA: an interior tile skips the
// damping and the Dirichlet tests altogether; a boundary tile uses per-row and
// per-column damping factors computed once instead of per point.
#pragma once
#include <cuda_runtime.h>

#include "kargs.h"

namespace fwi {
namespace st {

__device__ __forceinline__ float el(const float4& v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

// dh^2 * Laplacian at rows r..r+3 of one column from its x window W[0..8]
// (columns c-4..c+4 at rows r..r+3) and its z neighbours up (rows r-4..r-1)
// and dn (rows r+4..r+7).
__device__ __forceinline__ void lap_col(const float4* W, const float4& up, const float4& dn, float out[4]) {
    const float k0 = (float)(-2.0 * kFDM5), k1 = (float)kFDM4, k2 = (float)(-kFDM3), k3 = (float)kFDM2,
                k4 = (float)(-kFDM1);
    const float4 ow = W[4];
    const float z[12] = {up.x, up.y, up.z, up.w, ow.x, ow.y, ow.z, ow.w, dn.x, dn.y, dn.z, dn.w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float s1 = (el(W[3], e) + el(W[5], e)) + (z[e + 3] + z[e + 5]);
        const float s2 = (el(W[2], e) + el(W[6], e)) + (z[e + 2] + z[e + 6]);
        const float s3 = (el(W[1], e) + el(W[7], e)) + (z[e + 1] + z[e + 7]);
        const float s4 = (el(W[0], e) + el(W[8], e)) + (z[e + 0] + z[e + 8]);
        float l = k4 * s4;
        l = fmaf(k3, s3, l);
        l = fmaf(k2, s2, l);
        l = fmaf(k1, s1, l);
        out[e] = fmaf(k0, z[e + 4], l);
    }
}

// dh^2 * Laplacian at rows r..r+3 of the R consecutive columns c0..c0+R-1 of
// a shared tile stored column by column (LD floats per column, rows
// contiguous).  The R+8 float4 columns of the x stencil are read once into
// registers.  `own` returns the centre values.
template <int R>
__device__ __forceinline__ void lap_run_ld(const float* t, int LD, int r, int c0, float out[R][4], float4 own[R]) {
    float4 W[R + 8];
#pragma unroll
    for (int j = 0; j < R + 8; ++j) W[j] = *reinterpret_cast<const float4*>(t + (c0 - 4 + j) * LD + r);
#pragma unroll
    for (int m = 0; m < R; ++m) {
        const float* col = t + (c0 + m) * LD + r;
        const float4 up = *reinterpret_cast<const float4*>(col - 4);
        const float4 dn = *reinterpret_cast<const float4*>(col + 4);
        own[m] = W[m + 4];
        lap_col(W + m, up, dn, out[m]);
    }
}

// The same with the column pitch LD known at compile time.
template <int LD, int R>
__device__ __forceinline__ void lap_run(const float* t, int r, int c0, float out[R][4], float4 own[R]) {
    lap_run_ld<R>(t, LD, r, c0, out, own);
}

// Per-thread facts about its 4 rows i0..i0+3: update-region membership and
// the z damping profile.
struct Rows {
    float dz[4];
    unsigned inz, ok;  // bit e: row in the z damping band / inside 4..nzz-5
};

// Per-column facts.
struct Col {
    float dx;
    bool inx, ok;
};

__device__ __forceinline__ Rows rows_info(const float* __restrict__ b1d, int nb, int i0, int nzz) {
    Rows r;
    r.inz = 0;
    r.ok = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int i = i0 + e;
        const int iz = i < nb ? i : (i >= nzz - nb ? nzz - 1 - i : -1);
        r.dz[e] = (b1d && iz >= 0 && i < nzz) ? __ldg(b1d + iz) : 1.0f;
        if (b1d && iz >= 0 && i < nzz) r.inz |= 1u << e;
        if (i >= 4 && i < nzz - 4) r.ok |= 1u << e;
    }
    return r;
}

__device__ __forceinline__ Col col_info(const float* __restrict__ b1d, int nb, int j, int nxx) {
    Col c;
    const int jx = j < nb ? j : (j >= nxx - nb ? nxx - 1 - j : -1);
    c.inx = b1d && jx >= 0 && j >= 0 && j < nxx;
    c.dx = c.inx ? __ldg(b1d + jx) : 1.0f;
    c.ok = j >= 4 && j < nxx - 4;
    return c;
}

// The damper of get_boundary_damper (modeling.cu:355-402) from the two
// profiles: inside a corner b2d = (b1d[i] + b1d[j]) - 1, elsewhere the one
// profile that is not 1.
__device__ __forceinline__ float damp(const Rows& r, const Col& c, int e) {
    return ((r.inz >> e) & 1u) && c.inx ? (r.dz[e] + c.dx) - 1.0f : r.dz[e] * c.dx;
}

// The coefficient dt^2/dh^2 * v^2 of the four points, k2 * (v * v).
__device__ __forceinline__ float4 coef4(const float4& v, float k2) {
    return make_float4(k2 * (v.x * v.x), k2 * (v.y * v.y), k2 * (v.z * v.z), k2 * (v.w * v.w));
}

// One float4 of the forward update from the coefficients k4 = coef4(v, k2)
// (kernels that keep them resident call this directly).  EDGE: apply the
// Dirichlet zeroing; DAMP: apply the Cerjan damper.
template <bool DAMP, bool EDGE>
__device__ __forceinline__ float4 update4k(const float l[4], const float4& q, const float4& o, const float4& k4,
                                           const Rows& r, const Col& c) {
    float out[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float kk = el(k4, e);
        float res;
        if (DAMP) {
            const float d = damp(r, c, e);
            res = d * (kk * l[e] + 2.0f * el(q, e) - d * el(o, e));
        } else {
            res = kk * l[e] + 2.0f * el(q, e) - el(o, e);
        }
        if (EDGE) res = (c.ok && ((r.ok >> e) & 1u)) ? res : 0.0f;
        out[e] = res;
    }
    return make_float4(out[0], out[1], out[2], out[3]);
}

template <bool DAMP, bool EDGE>
__device__ __forceinline__ float4 update4(const float l[4], const float4& q, const float4& o, const float4& v,
                                          float k2, const Rows& r, const Col& c) {
    return update4k<DAMP, EDGE>(l, q, o, coef4(v, k2), r, c);
}

// One float4 of the backward step (cross_correlation / build_gradient,
// migration.cu:138-180, inversion.cu:405-444): the source field steps back,
// the receiver field forward, and image (Ps_new * Pr) or gradient
// (dt * Pr * lap(Psold) * v^2) and illumination (Ps_new^2) accumulate, only
// inside 4 <= i < nzz-4, 4 <= j < nxx-4 (colok and rows.ok).
struct Bwd4 {
    float4 ps, pr, a, b;
};
template <bool GRAD, bool EDGE>
__device__ __forceinline__ Bwd4 bwd_update4(const float ls[4], const float4& psold, const float lr[4],
                                            const float4& pr, const float4& ps, const float4& prold,
                                            const float4& vv, const float4& ga, const float4& gb, float dt2idh2,
                                            float dt, float idh2, const Rows& rows, bool colok) {
    float nps[4], npr[4], na[4], nb4[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const bool ok = !EDGE || (colok && ((rows.ok >> e) & 1u));
        const float v = el(vv, e);
        const float vp2 = v * v;
        const float k = dt2idh2 * vp2;
        const float s_new = k * ls[e] + 2.0f * el(psold, e) - el(ps, e);
        const float r_new = k * lr[e] + 2.0f * el(pr, e) - el(prold, e);
        nps[e] = ok ? s_new : 0.0f;
        npr[e] = ok ? r_new : 0.0f;
        const float prv = el(pr, e);
        const float da = GRAD ? dt * prv * (ls[e] * idh2) * vp2 : s_new * prv;
        const float db = s_new * s_new;
        na[e] = el(ga, e) + (ok ? da : 0.0f);
        nb4[e] = el(gb, e) + (ok ? db : 0.0f);
    }
    Bwd4 r;
    r.ps = make_float4(nps[0], nps[1], nps[2], nps[3]);
    r.pr = make_float4(npr[0], npr[1], npr[2], npr[3]);
    r.a = make_float4(na[0], na[1], na[2], na[3]);
    r.b = make_float4(nb4[0], nb4[1], nb4[2], nb4[3]);
    return r;
}

// Point injections of column j into rows z..z+3 (series sample `sample`).
__device__ __forceinline__ void inject4(const InjTable& inj, int sample, int col_off, int j, int z, float4& v) {
    if (sample < 0) return;
    const int kb = __ldg(inj.colptr + col_off + j), ke = __ldg(inj.colptr + col_off + j + 1);
    for (int k = kb; k < ke; ++k) {
        const int dz = __ldg(inj.z + k) - z;
        if (dz >= 0 && dz < 4) {
            const float amp = inj.scale * __ldg(inj.series + __ldg(inj.soff + k) + sample);
            if (dz == 0) v.x += amp;
            else if (dz == 1) v.y += amp;
            else if (dz == 2) v.z += amp;
            else v.w += amp;
        }
    }
}

// Whether columns [xa, xb) of a shot hold any injection point.
__device__ __forceinline__ bool has_points(const InjTable& inj, int col_off, int xa, int xb) {
    return xa < xb && __ldg(inj.colptr + col_off + xa) != __ldg(inj.colptr + col_off + xb);
}

// Tile classification: rows [z0, z0+h) x columns [x0, x0+w) (clipped to the grid).
__device__ __forceinline__ bool tile_inner(int z0, int h, int x0, int w, int nzz, int nxx) {
    return z0 >= 4 && z0 + h <= nzz - 4 && x0 >= 4 && x0 + w <= nxx - 4;
}
__device__ __forceinline__ bool tile_undamped(const float* b1d, int nb, int z0, int h, int x0, int w, int nzz,
                                              int nxx) {
    return !b1d || (z0 >= nb && z0 + h <= nzz - nb && x0 >= nb && x0 + w <= nxx - nb);
}

}  // namespace st
}  // namespace fwi
