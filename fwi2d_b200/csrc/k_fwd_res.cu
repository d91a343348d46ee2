// k_fwd_res.cu — every forward time level of a small survey with the wavefields
// resident in shared memory.
//
// Per point and level this is the forward step of the other kernels
// (compute_pressure + compute_seismogram, src/modeling/modeling.cu:301-353, in
// Jacobi order, st::update4k).  What changes is where the fields live: a
// B200's 148 SMs hold ~33 MB of shared memory, more than the two time levels
// of a survey such as 11 shots of 351 x 701 points (22 MB).  So instead of
// streaming every level's Q^t, Q^{t-1} and v through L2 / HBM,
//
//   * each CTA (one per SM, all co-resident through the cooperative launch)
//     owns one slab of one shot — a run of whole columns over the full
//     depth — and keeps Q^t (with a 4-column halo) and Q^{t-1} of its slab in
//     shared memory for the whole launch; Q^{t+1} overwrites Q^{t-1} in place
//     and the two buffers swap roles every level;
//   * the velocity enters once, as the per-point coefficients dt^2/dh^2 v^2,
//     which the thread that updates a point keeps in the SM's tensor memory
//     (TMEM: 256 KB per SM that a stencil leaves idle) and reads back with
//     tcgen05.ld every level, behind its shared-memory stencil loads — kept
//     in registers they would need a fully unrolled item loop whose code no
//     longer fits the instruction cache;
//   * the only traffic between CTAs is the halo: 4 columns on each side per
//     level, exchanged through a small global buffer (L2), not a grid
//     barrier.  Each 16-byte word carries two values and, twice, the level
//     that wrote them (the low-latency protocol of NCCL's LL transport), so
//     the reader polls the data itself: no fence, no flag, one L2 round trip
//     when the data is there.  A level computes the slab's interior first
//     (it needs no halo), then the edge columns, whose threads publish their
//     results at once; four exchange warps fetch the neighbours' edges of the
//     level before into the halo while the twelve compute warps finish the
//     interior, so the exchange hides behind it.
//
// The exchange buffer is double-buffered by level parity: a slab rewrites a
// parity slot two levels later, after it has read its neighbours' next
// level, which they published only after reading that slot.  It is zeroed
// before every launch (tag 0 is no level).  Every wait is bounded
// (tma::kSpinLimit polls); a wait that gives up raises *err and the CTA
// leaves the level loop (it has no asynchronous copies in flight; its TMEM
// is released), after which its neighbours' waits run out the same way.
#include <cuda_runtime.h>

#include "kargs.h"
#include "kernels.h"
#include "stencil.cuh"
#include "tma.cuh"

namespace fwi {

namespace {

constexpr int kRC = 384;        // compute threads (12 warps, 3 per SM sub-partition)
constexpr int kRX = 128;        // exchange threads (4 warps, 1 per sub-partition)
constexpr int kRT = kRC + kRX;
constexpr int kXB = 6;          // exchange words in flight per exchange thread
constexpr int kRecPerThread = 2;
constexpr int kMaxSrc = 16;     // injection points per slab

__device__ __forceinline__ void bar_arrive(int id, int n) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_sync(int id, int n) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
// Halo words {v0, tag, v1, tag}: two values of an edge column, each beside
// the level that wrote them.  Written and polled with 16-byte volatile
// accesses; a word counts only when both tags equal the level awaited (the
// 8-byte halves are each written at once), so no fence or flag is needed.
__device__ __forceinline__ void st_word(uint4* p, uint4 v) {
    asm volatile("st.volatile.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}
__device__ __forceinline__ uint4 ld_word(const uint4* p) {
    uint4 v;
    asm volatile("ld.volatile.global.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}

// Column of receiver / source entry r of a shot: colptr[col_off + x] <= r < colptr[col_off + x + 1].
__device__ __forceinline__ int entry_column(const int* colptr, int col_off, int lo, int hi, int r) {
    while (hi - lo > 1) {
        const int m = (lo + hi) >> 1;
        if (__ldg(colptr + col_off + m) <= r) lo = m;
        else hi = m;
    }
    return lo;
}

// Work of a slab per level, in 4 x 4 items (4 rows of a 4-column run): the
// interior runs 1..nruns-2 first — they read only the slab's own columns —
// then the two edge runs 0 and nruns-1, which read the halo and whose results
// the neighbours wait for.  Pass k of a compute thread holds interior item
// tid + k*kRC (k < pint) or edge item tid + (k-pint)*kRC.
struct Sched {
    int qg, nruns, nint, nedge, pint, pedge;
};
__host__ __device__ __forceinline__ Sched make_sched(int w, int ldz) {
    Sched sc;
    sc.qg = ldz / 4;
    sc.nruns = (w + 3) / 4;
    sc.nedge = (sc.nruns < 2 ? sc.nruns : 2) * sc.qg;
    sc.nint = sc.nruns * sc.qg - sc.nedge;
    sc.pint = (sc.nint + kRC - 1) / kRC;
    sc.pedge = (sc.nedge + kRC - 1) / kRC;
    return sc;
}
// Position (c0, gz) of pass k's item; false when the thread has none in that
// pass (the position is then run 0's, a safe place to read).
__device__ __forceinline__ bool item_of(const Sched& sc, int tid, int k, int* c0, int* gz) {
    int i, run;
    bool valid;
    if (k < sc.pint) {
        i = tid + k * kRC;
        valid = i < sc.nint;
        run = valid ? 1 + i / sc.qg : 0;
    } else {
        i = tid + (k - sc.pint) * kRC;
        valid = i < sc.nedge;
        run = (valid && i >= sc.qg) ? sc.nruns - 1 : 0;
    }
    *c0 = 4 * run;
    *gz = valid ? 4 * (i % sc.qg) : 0;
    return valid;
}

struct SrcList {
    int n;
    int lc[kMaxSrc], z[kMaxSrc];
    long long soff[kMaxSrc];
};

// ---- tensor memory: the per-point constants live there for the launch.
// Compute warp w reaches TMEM lanes 32*(w%4)..+31; warps w, w+4 and w+8
// take 160 of the 512 columns each; item k of a thread takes 32 columns:
// per item column m, its 4 coefficients dt^2/dh^2 v^2, then its 4 dampers.
constexpr int kTmemCols = 512;
constexpr int kItemCols = 32;
constexpr int kWarpCols = 160;
constexpr int kMaxPasses = kWarpCols / kItemCols;  // items per compute thread

__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr));
}
// The registers of a tcgen05.ld are defined only after the wait; passing them
// through it keeps every use behind it.
__device__ __forceinline__ void tmem_wait_ld32(uint32_t (&r)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_st32(uint32_t addr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};"
        ::"r"(addr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]),
        "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
        "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Q^{t+1} of one 4 x 4 item, rows gz..gz+3 of slab columns c0..c0+ncol-1:
// the Laplacian of Q^t in A column by column from the item's x window, Q^{t-1}
// in B (pointwise, overwritten) and the item's constants kr (per column:
// coefficients, dampers) from TMEM.  Items of an edge run also publish their
// results to pub_a / pub_b (a side of the slab's exchange words, or NULL).  One expression serves every point: the
// damped update of the other kernels, new = d * (kk * L + 2 q - d * old), with
// d = 1 outside the ABC band (multiplications by 1 are exact) and d = 0 on the
// Dirichlet rim.
__device__ __forceinline__ void res_item(const FwdResArgs& a, const float* A, float* B, int lds, int c0, int gz,
                                         int ncol, bool valid, uint32_t tcol, const SrcList& src, int sample,
                                         uint4* pub_a, uint4* pub_b, unsigned tag) {
    uint32_t kr[32];
    __syncwarp();
    tmem_ld32(tcol, kr);
    const float* t = A + (c0 + 4) * lds + 4 + gz;  // Q^t at (gz, c0)
    float4 W[12];
#pragma unroll
    for (int j = 0; j < 12; ++j) W[j] = *reinterpret_cast<const float4*>(t + (j - 4) * lds);
    __syncwarp();
    tmem_wait_ld32(kr);
    if (!valid) return;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        if (m >= ncol) break;
        const float* col = t + m * lds;
        float l[4];
        st::lap_col(W + m, *reinterpret_cast<const float4*>(col - 4), *reinterpret_cast<const float4*>(col + 4), l);
        float* po = B + (c0 + m + 4) * lds + 4 + gz;
        const float4 oo = *reinterpret_cast<const float4*>(po);
        float res[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float kk = __uint_as_float(kr[8 * m + e]);
            const float d = __uint_as_float(kr[8 * m + 4 + e]);
            res[e] = d * (kk * l[e] + 2.0f * st::el(W[m + 4], e) - d * st::el(oo, e));
        }
        float4 out = make_float4(res[0], res[1], res[2], res[3]);
        if (sample >= 0) {
            for (int k = 0; k < src.n; ++k) {
                const int dz = src.z[k] - gz;
                if (src.lc[k] != c0 + m || dz < 0 || dz >= 4) continue;
                const float amp = a.inj.scale * __ldg(a.inj.series + src.soff[k] + sample);
                if (dz == 0) out.x += amp;
                else if (dz == 1) out.y += amp;
                else if (dz == 2) out.z += amp;
                else out.w += amp;
            }
        }
        *reinterpret_cast<float4*>(po) = out;
        // an edge column: also to the neighbour, as two tagged words
        const size_t j = (size_t)(m * a.ldz + gz) / 2;
        const uint4 w0 = make_uint4(__float_as_uint(out.x), tag, __float_as_uint(out.y), tag);
        const uint4 w1 = make_uint4(__float_as_uint(out.z), tag, __float_as_uint(out.w), tag);
        if (pub_a) {
            st_word(pub_a + j, w0);
            st_word(pub_a + j + 1, w1);
        }
        if (pub_b) {
            st_word(pub_b + j, w0);
            st_word(pub_b + j + 1, w1);
        }
    }
}

__global__ void __launch_bounds__(kRT, 1) fwd_res_kernel(const FwdResArgs a) {
    extern __shared__ __align__(16) float smem[];
    __shared__ SrcList src;
    __shared__ int abort_flag;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_pos[kMaxPasses * kRC];  // per pass and compute thread: item position, < 0: none
    const int tid = threadIdx.x, warp = tid >> 5;
    const ResSlab sl = a.slabs[blockIdx.x];
    const ShotDesc sd = a.shots[sl.s];
    const int lds = a.ldz + 8;  // stored column: 4 zero rows, ldz rows, 4 zero rows
    const int qg = a.ldz / 4;   // 4-row groups per column
    const Sched sc = make_sched(sl.w, a.ldz);
    const int passes = sc.pint + sc.pedge;
    // the exchange warps fetch the halo during the last two interior passes:
    // the neighbours published it as the level began, so by then it has as a
    // rule landed in L2 and one round of loads brings it, without polling
    const int fetch_after = sc.pint > 2 ? sc.pint - 2 : 0;
    const long long so = (long long)sl.s * a.fstride;
    // the two field buffers, as offsets into smem (the Q^t / Q^{t-1} roles
    // swap every level; offsets keep every access a shared-memory one)
    int oa = 0, ob = (a.wmax + 8) * lds;
    float* buf0 = smem + oa;
    float* buf1 = smem + ob;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tma::smem_addr(&tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        tc_fence_before();
    }
    // ---- set-up: zero both buffers, load Q^t (own columns + halo) and Q^{t-1}
    {
        float4* s4 = reinterpret_cast<float4*>(smem);
        const int n4 = 2 * (a.wmax + 8) * lds / 4;
        for (int i = tid; i < n4; i += kRT) s4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (tid == 0) abort_flag = 0;
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    for (int i = tid; i < (sl.w + 8) * qg; i += kRT) {
        const int c = i / qg - 4, q = i - (i / qg) * qg;
        const int gx = sl.x0 + c;
        if (gx < 0 || gx >= sd.nxx) continue;
        const size_t g = (size_t)so + (size_t)gx * a.ldz + 4 * q;
        *reinterpret_cast<float4*>(buf0 + (c + 4) * lds + 4 + 4 * q) =
            __ldg(reinterpret_cast<const float4*>(a.in_cur + g));
        if (c >= 0 && c < sl.w)
            *reinterpret_cast<float4*>(buf1 + (c + 4) * lds + 4 + 4 * q) =
                __ldg(reinterpret_cast<const float4*>(a.in_old + g));
    }
    // receivers of the slab's columns (kRecPerThread per compute thread)
    int rec_idx[kRecPerThread];
    long long rec_off[kRecPerThread];
    float rec_d[kRecPerThread];
    const int rkb = __ldg(a.rec.colptr + sd.col_off + sl.x0);
    const int rke = a.seis ? __ldg(a.rec.colptr + sd.col_off + sl.x0 + sl.w) : rkb;
#pragma unroll
    for (int j = 0; j < kRecPerThread; ++j) {
        const int r = rkb + tid + j * kRC;
        rec_idx[j] = -1;
        rec_off[j] = 0;
        rec_d[j] = 0.0f;
        if (tid < kRC && r < rke) {
            const int x = entry_column(a.rec.colptr, sd.col_off, sl.x0, sl.x0 + sl.w, r);
            const int z = __ldg(a.rec.z + r);
            rec_idx[j] = (x - sl.x0 + 4) * lds + 4 + z;
            rec_off[j] = __ldg(a.rec.soff + r);
            rec_d[j] = a.b1d ? st::damp(st::rows_info(a.b1d, a.nb, z, a.nzz), st::col_info(a.b1d, a.nb, x, sd.nxx), 0)
                             : 1.0f;
        }
    }
    // injection points of the slab's columns
    const int skb = __ldg(a.inj.colptr + sd.col_off + sl.x0);
    const int ske = __ldg(a.inj.colptr + sd.col_off + sl.x0 + sl.w);
    if (tid == 0) src.n = ske - skb;
    if (tid < ske - skb && tid < kMaxSrc) {
        const int r = skb + tid;
        src.lc[tid] = entry_column(a.inj.colptr, sd.col_off, sl.x0, sl.x0 + sl.w, r) - sl.x0;
        src.z[tid] = __ldg(a.inj.z + r);
        src.soff[tid] = __ldg(a.inj.soff + r);
    }
    // slabs the host planned outside these tables never run (the same test on every thread)
    const bool fits = rke - rkb <= kRecPerThread * kRC && ske - skb <= kMaxSrc && passes <= kMaxPasses &&
                      a.ldz % 2 == 0;
    if (!fits && tid == 0) atomicExch(a.err, 1);
    // the thread's TMEM columns: lanes of its warp quarter, its half of the columns
    const uint32_t tbase = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * kWarpCols);
    if (fits && tid < kRC) {
        // the coefficients dt^2/dh^2 v^2 and dampers of the thread's items, once
        // for the launch: d = the ABC damper (1 without ABC), 0 outside the
        // update region 4 <= i < nzz-4, 4 <= j < nxx-4
        const float* vb = a.vel + (size_t)sl.s * a.vel_stride;
        for (int k = 0; k < passes; ++k) {
            int c0 = 0, gz = 0;
            const bool valid = item_of(sc, tid, k, &c0, &gz);
            s_pos[k * kRC + tid] = (valid ? 0 : (int)0x80000000) | (c0 << 16) | gz;
            const st::Rows rows = st::rows_info(a.b1d, a.nb, gz, a.nzz);
            uint32_t kr[32];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int gx = sl.x0 + c0 + m;
                const bool col_in = valid && c0 + m < sl.w;
                const float4 k4 =
                    col_in ? st::coef4(__ldg(reinterpret_cast<const float4*>(vb + (size_t)(gx + sd.vel_col) * a.ldz + gz)),
                                       a.dt2idh2)
                           : make_float4(0.f, 0.f, 0.f, 0.f);
                const st::Col col = st::col_info(a.b1d, a.nb, gx, sd.nxx);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const bool ok = col_in && col.ok && ((rows.ok >> e) & 1u);
                    kr[8 * m + e] = __float_as_uint(ok ? st::el(k4, e) : 0.0f);
                    kr[8 * m + 4 + e] = __float_as_uint(ok ? st::damp(rows, col, e) : 0.0f);
                }
            }
            __syncwarp();
            tmem_st32(tbase + kItemCols * k, kr);
        }
        tmem_wait_st();
    }
    __syncthreads();

    bool done = !fits;
    for (int t = a.t_begin; t < a.t_end && !done; ++t) {
        float* A = smem + oa;  // Q^t (stencil)
        float* B = smem + ob;  // Q^{t-1}, then Q^{t+1}
        // level L computes Q^{t+1} and publishes its edges with tag L + 1; the
        // halo of Q^t came with tag L (from the field buffers when L = 0)
        const unsigned lv = (unsigned)(t - a.t_begin);
        const int nw = 2 * a.ldz;  // exchange words per side: 4 columns, 2 values a word
        if (tid < kRC) {
            // ---------- compute warps
            if (a.seis && t > a.tlag) {
#pragma unroll
                for (int j = 0; j < kRecPerThread; ++j)
                    if (rec_idx[j] >= 0) a.seis[rec_off[j] + (t - a.tlag)] = rec_d[j] * A[rec_idx[j]];
            }
            const int sample = (t + 1 < a.nt) ? t + 1 : -1;
            uint4* mine = a.xbuf + ((size_t)((lv + 1) & 1u) * a.nslab + blockIdx.x) * 2 * nw;
            for (int k = 0; k < passes; ++k) {
                if (k == fetch_after) bar_arrive(2, kRT);  // the exchange warps may start fetching
                if (k == sc.pint) bar_sync(1, kRT);        // the halo of Q^t is in A
                const int pos = s_pos[k * kRC + tid];
                const bool valid = pos >= 0;
                const int c0 = (pos >> 16) & 0x7fff, gz = pos & 0xffff;
                uint4* pa = (k >= sc.pint && sl.left >= 0 && c0 == 0) ? mine : nullptr;
                uint4* pb = (k >= sc.pint && sl.right >= 0 && c0 + 4 >= sl.w) ? mine + nw : nullptr;
                res_item(a, A, B, lds, c0, gz, min(4, sl.w - c0), valid, tbase + kItemCols * k, src, sample, pa, pb,
                         lv + 1);
            }
            if (sc.pedge == 0) bar_sync(1, kRT);
        } else {
            // ---------- exchange warps: the neighbours' edges of Q^t (tag L)
            // into the halo columns of A, while the interior is computed.
            // Word w < nw: the left neighbour's right edge -> columns -4..-1;
            // w >= nw: the right neighbour's left edge -> columns w..w+3.
            bar_sync(2, kRT);
            const int x = tid - kRC;
            const size_t slot = lv & 1u;
            const uint4* from_left = a.xbuf + (slot * a.nslab + (sl.left >= 0 ? sl.left : 0)) * 2 * nw + nw;
            const uint4* from_right = a.xbuf + (slot * a.nslab + (sl.right >= 0 ? sl.right : 0)) * 2 * nw;
            bool ok = true;
            for (int base = x; lv > 0 && base < 2 * nw && ok; base += kRX * kXB) {
                uint4 v[kXB];
                unsigned pending = 0;
#pragma unroll
                for (int i = 0; i < kXB; ++i) {
                    const int w = base + i * kRX;
                    const bool left = w < nw;
                    if (w >= 2 * nw || (left ? sl.left : sl.right) < 0) continue;
                    v[i] = ld_word(left ? from_left + w : from_right + (w - nw));
                    if (v[i].y != lv || v[i].w != lv) pending |= 1u << i;
                }
                // poll the first pending word only, backing off, so that the
                // polling takes little of the L2 and LSU bandwidth the compute
                // warps use; once it has arrived, the others have as a rule
                unsigned nap = 128;
                for (uint32_t spin = 0; pending && spin < tma::kSpinLimit; ++spin) {
                    __nanosleep(nap);
                    nap = nap < 512 ? 2 * nap : 512;
                    const int first = __ffs(pending) - 1;
#pragma unroll
                    for (int i = 0; i < kXB; ++i) {
                        if (i < first || !((pending >> i) & 1u)) continue;
                        const int w = base + i * kRX;
                        v[i] = ld_word(w < nw ? from_left + w : from_right + (w - nw));
                        if (v[i].y == lv && v[i].w == lv) pending &= ~(1u << i);
                        else break;
                    }
                }
                ok = pending == 0;
#pragma unroll
                for (int i = 0; i < kXB; ++i) {
                    const int w = base + i * kRX;
                    const bool left = w < nw;
                    if (!ok || w >= 2 * nw || (left ? sl.left : sl.right) < 0) continue;
                    const int vv = 2 * (left ? w : w - nw), c = vv / a.ldz, z = vv - (vv / a.ldz) * a.ldz;
                    const int col = left ? c - 4 : sl.w + c;
                    *reinterpret_cast<float2*>(A + (col + 4) * lds + 4 + z) =
                        make_float2(__uint_as_float(v[i].x), __uint_as_float(v[i].z));
                }
            }
            if (!ok) {
                atomicExch(a.err, 1);
                abort_flag = 1;
            }
            bar_arrive(1, kRT);
        }
        __syncthreads();
        done = abort_flag != 0;
        const int o = oa;
        oa = ob;
        ob = o;
    }

    if (fits && !abort_flag) {
        // ---- write back the own columns: Q^t and Q^{t-1}
        const float* A = smem + oa;
        const float* B = smem + ob;
        for (int i = tid; i < sl.w * qg; i += kRT) {
            const int c = i / qg, q = i - (i / qg) * qg;
            const size_t g = (size_t)so + (size_t)(sl.x0 + c) * a.ldz + 4 * q;
            *reinterpret_cast<float4*>(a.out_cur + g) =
                *reinterpret_cast<const float4*>(A + (c + 4) * lds + 4 + 4 * q);
            *reinterpret_cast<float4*>(a.out_old + g) =
                *reinterpret_cast<const float4*>(B + (c + 4) * lds + 4 + 4 * q);
        }
    }
    // ---- release the tensor memory on every path
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}

// More than half of an SM's shared memory: one CTA per SM, so that the CTA
// can take all 512 TMEM columns.
constexpr size_t kMinSmem = 116 * 1024;

cudaError_t res_configure(size_t smem, int* ctas) {
    smem = smem < kMinSmem ? kMinSmem : smem;
    cudaError_t e = cudaFuncSetAttribute(fwd_res_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fwd_res_kernel, kRT, smem);
    return e;
}

cudaError_t res_launch(const FwdResArgs& a, size_t smem, cudaStream_t st) {
    smem = smem < kMinSmem ? kMinSmem : smem;
    void* args[] = {const_cast<FwdResArgs*>(&a)};
    return cudaLaunchCooperativeKernel((const void*)fwd_res_kernel, dim3(a.nslab), dim3(kRT), args, smem, st);
}

}  // namespace

int fwd_res_threads() { return kRC; }
int fwd_res_max_rec() { return kRecPerThread * kRC; }
int fwd_res_max_src() { return kMaxSrc; }
bool fwd_res_fits(int w, int ldz) {
    const Sched sc = make_sched(w, ldz);
    return sc.pint + sc.pedge <= kMaxPasses;
}

size_t fwd_res_smem(int wmax, int ldz) {
    const size_t need = (size_t)2 * (wmax + 8) * (ldz + 8) * sizeof(float);
    return need < kMinSmem ? kMinSmem : need;
}

size_t fwd_res_static_smem() {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fwd_res_kernel) != cudaSuccess) {
        cudaGetLastError();
        return sizeof(SrcList) + 64;
    }
    return fa.sharedSizeBytes;
}

cudaError_t fwd_res_configure(size_t smem, int* ctas_per_sm) { return res_configure(smem, ctas_per_sm); }

cudaError_t launch_fwd_res(const FwdResArgs& a, size_t smem, cudaStream_t st) { return res_launch(a, smem, st); }

}  // namespace fwi
