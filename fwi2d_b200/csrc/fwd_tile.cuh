// fwd_tile.cuh — tile geometry, tile metadata and the per-tile compute passes
// shared by the forward TMA kernels (k_fwd_tma.cu: one or two time levels per
// launch; k_fwd_loop.cu: every time level in one cooperative launch).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "kargs.h"
#include "stencil.cuh"
#include "tma.cuh"

namespace fwi {
namespace ft {
constexpr int kTZ = 128;   // output rows per tile
constexpr int kNC = 256;   // consumer threads (8 warps) per CTA
constexpr int kNT = kNC + 32;  // + one producer warp

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

// Per-tile facts the producer warp gathers (global loads off the consumers'
// critical path) and publishes next to the tile's shared-memory stage.
struct TileMeta {
    int s, x0, z0, nxx, col_off;
    int has_src;         // the tile or its 4-cell ring holds a source point
    int rec_kb, rec_ke;  // receiver entries of the tile's columns
};

// Everything a pass over one staged tile needs.
struct Tile {
    const float* cur;   // Q^t with an H-cell halo
    const float* old;   // Q^{t-1} with an (H-4)-cell halo
    const float* vel;   // v with an (H-4)-cell halo
    float* mid;         // Q^{t+1} with a 4-cell ring (T = 2)
    TileInfo ti;
    int nxx, col_off;
    bool has_src;
};

// T = 2: Q^{t+1} on the tile and its 4-cell ring, runs of 4 columns.
template <int T, int TX, bool DAMP, bool EDGE>
__device__ __forceinline__ void mid_pass(const FwdTmaArgs& a, const Tile& t) {
    using G = Geom<T, TX>;
    constexpr int QZ = G::MZ / 4;
    constexpr int RUNS = G::MX / 4;
    for (int w = threadIdx.x; w < QZ * RUNS; w += kNC) {
        const int q = w % QZ, c0 = (w / QZ) * 4;
        const int gz = t.ti.z0 - 4 + 4 * q;
        const st::Rows rows = st::rows_info(DAMP ? a.b1d : nullptr, a.nb, gz, a.nzz);
        float l[4][4];
        float4 qq[4];
        st::lap_run<G::CZ, 4>(t.cur, 4 * q + 4, c0 + 4, l, qq);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int c = c0 + m, gx = t.ti.x0 - 4 + c;
            const float4 oo = *reinterpret_cast<const float4*>(t.old + c * G::PZ + 4 * q);
            const float4 vv = *reinterpret_cast<const float4*>(t.vel + c * G::PZ + 4 * q);
            const st::Col col =
                (DAMP || EDGE) ? st::col_info(DAMP ? a.b1d : nullptr, a.nb, gx, t.nxx) : st::Col{1.0f, false, true};
            float4 out = st::update4<DAMP, EDGE>(l[m], qq[m], oo, vv, a.dt2idh2, rows, col);
            if (t.has_src && gx >= 0 && gx < t.nxx) st::inject4(a.inj, a.sample1, t.col_off, gx, gz, out);
            *reinterpret_cast<float4*>(t.mid + c * G::MZ + 4 * q) = out;
        }
    }
}

// Last level of the launch on the tile: thread (lane, warp) owns rows
// z0+4*lane .. +3 of the warp's TX/8 consecutive columns.
template <int T, int TX, bool DAMP, bool EDGE>
__device__ __forceinline__ void final_pass(const FwdTmaArgs& a, const Tile& t) {
    using G = Geom<T, TX>;
    constexpr int CPW = TX / 8;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int z = t.ti.z0 + 4 * lane;
    if (z >= a.ldz) return;
    const st::Rows rows = st::rows_info(DAMP ? a.b1d : nullptr, a.nb, z, a.nzz);
    const int c0 = warp * CPW;
    float l[CPW][4];
    float4 qq[CPW];
    if (T == 2) st::lap_run<G::MZ, CPW>(t.mid, 4 * lane + 4, c0 + 4, l, qq);
    else st::lap_run<G::CZ, CPW>(t.cur, 4 * lane + 4, c0 + 4, l, qq);
#pragma unroll
    for (int m = 0; m < CPW; ++m) {
        const int c = c0 + m;
        const int gx = t.ti.x0 + c;
        if (gx >= t.nxx) break;
        const size_t goff = (size_t)t.ti.s * a.fstride + (size_t)gx * a.ldz + z;
        if (T == 2) *reinterpret_cast<float4*>(a.out1 + goff) = qq[m];  // Q^{t+1} on the tile
        const float4 oo = (T == 2) ? *reinterpret_cast<const float4*>(t.cur + (c + 8) * G::CZ + 4 * lane + 8)
                                   : *reinterpret_cast<const float4*>(t.old + c * G::PZ + 4 * lane);
        const float4 vv =
            *reinterpret_cast<const float4*>(t.vel + (c + G::H - 4) * G::PZ + 4 * lane + (G::H - 4));
        const st::Col col =
            (DAMP || EDGE) ? st::col_info(DAMP ? a.b1d : nullptr, a.nb, gx, t.nxx) : st::Col{1.0f, false, true};
        float4 out = st::update4<DAMP, EDGE>(l[m], qq[m], oo, vv, a.dt2idh2, rows, col);
        if (t.has_src) st::inject4(a.inj, T == 2 ? a.sample2 : a.sample1, t.col_off, gx, z, out);
        *reinterpret_cast<float4*>((T == 2 ? a.out2 : a.out1) + goff) = out;
    }
}

__device__ __forceinline__ void consumer_barrier() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

}  // namespace ft
}  // namespace fwi
