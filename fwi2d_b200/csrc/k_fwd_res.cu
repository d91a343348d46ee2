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
//     barrier.  Each value travels in a 64-bit half beside the level that
//     wrote it (the low-latency protocol of NCCL's LL transport), so the
//     reader checks the data itself: no fence and no flag.  A level computes
//     the slab's two edge runs first and their threads publish the results
//     at once; then the interior, during whose last two passes every thread
//     starts asynchronous copies (cp.async, L2 -> shared memory) of its share
//     of the neighbours' edges, published most of a level earlier; after the
//     last pass it checks the levels and unpacks them into the halo.  The copies never
//     stall the compute warps (loads issued to L2 by warps of their own,
//     queued behind the compute warps' shared-memory traffic, took longer
//     than the whole interior), and the only barrier is the one per level.
//
// The exchange buffer is double-buffered by level parity: a slab rewrites a
// parity slot two levels later, after it has read its neighbours' next
// level, which they published only after reading that slot.  It is zeroed
// before every launch (level 0 is no level).  Every wait is bounded
// (tma::kSpinLimit polls); a wait that gives up raises *err and the CTA
// leaves the level loop (with no asynchronous copy in flight and its TMEM
// released), after which its neighbours' waits run out the same way.
//
// Failure drill: a second instantiation (DRILL, generic column pitch) takes
// the wait limit from a.spin, gives a poll up as soon as *err is raised
// (checked every 32nd poll) and lets slab a.stall publish its halo words into
// a spare area that nobody reads, so its neighbours' polls run out.  Only
// contexts given the test keys launch it: the production instantiations keep
// the constant limit, whose code the level loop's schedule was tuned with.
#include <cuda_runtime.h>

#include "kargs.h"
#include "kernels.h"
#include "stencil.cuh"
#include "tma.cuh"

namespace fwi {

namespace {

constexpr int kRC = 384;        // threads (12 warps, 3 per SM sub-partition)
constexpr int kRT = kRC;
constexpr int kRecPerThread = 2;
constexpr int kMaxXW = 4;       // halo words per thread and level: 4 ldz <= kMaxXW * kRT
constexpr int kMaxSrc = 16;     // injection points per slab

// Halo words: two values of an edge column, each in a 64-bit half beside the
// level that wrote it (value bits | level << 32).  A 64-bit access is
// single-copy atomic, so a half whose level is the one awaited holds that
// level's value: the reader polls the data itself, with no fence and no flag.
// Relaxed gpu-scope accesses: they reach L2 and may be pipelined.
__device__ __forceinline__ void st_word(ulonglong2* p, float v0, float v1, unsigned tag) {
    const unsigned long long t = (unsigned long long)tag << 32;
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(t | __float_as_uint(v0)),
                 "l"(t | __float_as_uint(v1))
                 : "memory");
}
__device__ __forceinline__ ulonglong2 ld_word(const ulonglong2* p) {
    ulonglong2 v;
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool word_is(const ulonglong2& v, unsigned tag) {
    return (unsigned)(v.x >> 32) == tag && (unsigned)(v.y >> 32) == tag;
}
// 16-byte asynchronous copy L2 -> shared memory (bypassing L1)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tma::smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
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
// two edge runs 0 and nruns-1 first — they read the halo and the neighbours
// wait for their results — then the interior runs 1..nruns-2, which read only
// the slab's own columns, in one stream: pass k of a thread holds item
// tid + k*kRC, so no pass is left part-empty by the edges.
struct Sched {
    int qg, nruns, nint, nedge, passes;
};
__host__ __device__ __forceinline__ Sched make_sched(int w, int ldz) {
    Sched sc;
    sc.qg = ldz / 4;
    sc.nruns = (w + 3) / 4;
    sc.nedge = (sc.nruns < 2 ? sc.nruns : 2) * sc.qg;
    sc.nint = sc.nruns * sc.qg - sc.nedge;
    sc.passes = (sc.nedge + sc.nint + kRC - 1) / kRC;
    return sc;
}
// Position (c0, gz) of pass k's item; false when the thread has none in that
// pass (the position is then run 0's, a safe place to read).
__device__ __forceinline__ bool item_of(const Sched& sc, int tid, int k, int* c0, int* gz) {
    const int i = tid + k * kRC;
    int run = 0, q = 0;
    const bool valid = i < sc.nedge + sc.nint;
    if (valid && i < sc.nedge) {
        run = i >= sc.qg ? sc.nruns - 1 : 0;
        q = i % sc.qg;
    } else if (valid) {
        run = 1 + (i - sc.nedge) / sc.qg;
        q = (i - sc.nedge) % sc.qg;
    }
    *c0 = 4 * run;
    *gz = 4 * q;
    return valid;
}

struct SrcList {
    int n;
    int lc[kMaxSrc], z[kMaxSrc];
    long long soff[kMaxSrc];
};

// ---- tensor memory: the per-point constants live there for the launch.
// Warp w reaches TMEM lanes 32*(w%4)..+31; warps w, w+4 and w+8
// take 160 of the 512 columns each; item k of a thread takes 32 columns:
// per item column m, its 4 negated coefficients -dt^2/dh^2 v^2, then its 4 dampers.
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

// ---- packed FP32 pairs (sm_100 FADD2 / FMUL2 / FFMA2): two IEEE float
// operations per instruction, each rounded as its scalar form, so the pair
// versions below give the bits of the scalar arithmetic in half the issue
// slots.
typedef unsigned long long f2;
__device__ __forceinline__ f2 pk(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 upk(f2 v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// dh^2 * Laplacian at rows r..r+3 of one column, as st::lap_col (the same
// sums in the same order) on the point pairs (r, r+1) and (r+2, r+3).  z pairs
// aligned with a float4 are A0..A5 (up, own, dn halves); the pairs straddling
// two halves are S0..S4.
__device__ __forceinline__ void lap_col2(const float4* W, const float4& up, const float4& dn, f2 out[2]) {
    const f2 k0 = pk((float)(-2.0 * kFDM5), (float)(-2.0 * kFDM5)), k1 = pk((float)kFDM4, (float)kFDM4),
             k2 = pk((float)(-kFDM3), (float)(-kFDM3)), k3 = pk((float)kFDM2, (float)kFDM2),
             k4 = pk((float)(-kFDM1), (float)(-kFDM1));
    const float4 ow = W[4];
    const f2 A0 = pk(up.x, up.y), A1 = pk(up.z, up.w), A2 = pk(ow.x, ow.y), A3 = pk(ow.z, ow.w), A4 = pk(dn.x, dn.y),
             A5 = pk(dn.z, dn.w);
    const f2 S0 = pk(up.y, up.z), S1 = pk(up.w, ow.x), S2 = pk(ow.y, ow.z), S3 = pk(ow.w, dn.x), S4 = pk(dn.y, dn.z);
    // z sums per pair and k = 1..4; centres
    const f2 zs[2][4] = {{add2(S1, S2), add2(A1, A3), add2(S0, S3), add2(A0, A4)},
                         {add2(S2, S3), add2(A2, A4), add2(S1, S4), add2(A1, A5)}};
    const f2 ctr[2] = {A2, A3};
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        f2 sk[4];
#pragma unroll
        for (int k = 1; k <= 4; ++k) {
            const f2 xm = p == 0 ? pk(W[4 - k].x, W[4 - k].y) : pk(W[4 - k].z, W[4 - k].w);
            const f2 xp = p == 0 ? pk(W[4 + k].x, W[4 + k].y) : pk(W[4 + k].z, W[4 + k].w);
            sk[k - 1] = add2(add2(xm, xp), zs[p][k - 1]);
        }
        f2 l = mul2(k4, sk[3]);
        l = fma2(k3, sk[2], l);
        l = fma2(k2, sk[1], l);
        l = fma2(k1, sk[0], l);
        out[p] = fma2(k0, ctr[p], l);
    }
}

// Q^{t+1} of one 4 x 4 item, rows gz..gz+3 of slab columns c0..c0+3 (a
// partial last run of a shot computes zeros past its edge, d = 0 there): the
// Laplacian of Q^t in A column by column from the item's x window, Q^{t-1} in
// B (pointwise, overwritten) and the item's constants kr from TMEM (per
// column: the negated coefficients -kk, then the dampers d).  One expression
// serves every point, the damped update of the other kernels
//     new = d * (kk * L + 2 q - d * old)
// with d = 1 outside the ABC band (multiplications by 1 are exact) and d = 0
// on the Dirichlet rim.  It is evaluated on point pairs with the same
// roundings as its scalar contraction u = fma(kk, L, 2q), new = d * fma(-d,
// old, u): nu = fma(-kk, L, -2q) = -u and fma(d, old, nu) = -fma(-d, old, u)
// exactly, and new = (-d) * that.  Items of an edge run also publish their
// results to pub_a / pub_b (a side of the slab's exchange words, or NULL).
__device__ __forceinline__ void res_item(const FwdResArgs& a, const float* A, float* B, int lds, int c0, int gz,
                                         bool valid, bool src_here, uint32_t tcol, const SrcList& src, int sample,
                                         ulonglong2* pub_a, ulonglong2* pub_b, unsigned tag) {
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
    const f2 m2 = pk(-2.0f, -2.0f), m1 = pk(-1.0f, -1.0f);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const float* col = t + m * lds;
        f2 l[2];
        lap_col2(W + m, *reinterpret_cast<const float4*>(col - 4), *reinterpret_cast<const float4*>(col + 4), l);
        float* po = B + (c0 + m + 4) * lds + 4 + gz;
        const float4 oo = *reinterpret_cast<const float4*>(po);
        float2 res[2];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            // -(kk L + 2 q), d old - (kk L + 2 q), then d (kk L + 2 q - d old) = -d * that
            const f2 nkk = pk(__uint_as_float(kr[8 * m + 2 * p]), __uint_as_float(kr[8 * m + 2 * p + 1]));
            const f2 d = pk(__uint_as_float(kr[8 * m + 4 + 2 * p]), __uint_as_float(kr[8 * m + 5 + 2 * p]));
            const f2 q = p == 0 ? pk(W[m + 4].x, W[m + 4].y) : pk(W[m + 4].z, W[m + 4].w);
            const f2 o = p == 0 ? pk(oo.x, oo.y) : pk(oo.z, oo.w);
            const f2 nu = fma2(nkk, l[p], mul2(q, m2));
            res[p] = upk(mul2(mul2(d, m1), fma2(d, o, nu)));
        }
        float4 out = make_float4(res[0].x, res[0].y, res[1].x, res[1].y);
        if (src_here && sample >= 0) {
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
        const int j = m * (a.ldz >> 1) + (gz >> 1);
        if (pub_a) {
            st_word(pub_a + j, out.x, out.y, tag);
            st_word(pub_a + j + 1, out.z, out.w, tag);
        }
        if (pub_b) {
            st_word(pub_b + j, out.x, out.y, tag);
            st_word(pub_b + j + 1, out.z, out.w, tag);
        }
    }
}

// LDS: the stored column pitch ldz + 8 when known at compile time (every
// shared-memory offset of the stencil becomes an immediate), 0 for any ldz.
template <int LDS, bool DRILL>
__global__ void __launch_bounds__(kRT, 1) fwd_res_kernel(const FwdResArgs a) {
    extern __shared__ __align__(16) float smem[];
    __shared__ SrcList src;
    __shared__ int abort_flag;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_pos[kMaxPasses * kRC];  // per pass and compute thread: item position, < 0: none
    const int tid = threadIdx.x, warp = tid >> 5;
    const ResSlab sl = a.slabs[blockIdx.x];
    const ShotDesc sd = a.shots[sl.s];
    const int lds = LDS ? LDS : a.ldz + 8;  // stored column: 4 zero rows, ldz rows, 4 zero rows
    const int qg = a.ldz / 4;   // 4-row groups per column
    const Sched sc = make_sched(sl.w, a.ldz);
    const int passes = sc.passes;
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
                      4 * a.ldz <= kMaxXW * kRT;
    if (!fits && tid == 0) atomicExch(a.err, 1);
    __syncthreads();  // the source list is complete
    // this thread's halo words, w = tid + i*kRT of the 4 ldz: w < 2 ldz from the left
    // neighbour's right side (-> columns -4..-1), the others from the right
    // neighbour's left side (-> columns w..w+3); xdst: float offset of the two
    // values in a field buffer, -1 for none
    const int nw = 2 * a.ldz;  // words per side: 4 columns, 2 values a word
    int xdst[kMaxXW];
#pragma unroll
    for (int i = 0; i < kMaxXW; ++i) {
        const int w = tid + i * kRT;
        const bool left = w < nw;
        xdst[i] = -1;
        if (w < 2 * nw && (left ? sl.left : sl.right) >= 0) {
            const int v = 2 * (left ? w : w - nw), c = v / a.ldz, z = v - c * a.ldz;
            xdst[i] = ((left ? c - 4 : sl.w + c) + 4) * lds + 4 + z;
        }
    }
    // the thread's TMEM columns: lanes of its warp's quarter, its warp's third of the columns
    const uint32_t tbase = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * kWarpCols);
    if (fits && tid < kRC) {
        // the coefficients dt^2/dh^2 v^2 and dampers of the thread's items, once
        // for the launch: d = the ABC damper (1 without ABC), 0 outside the
        // update region 4 <= i < nzz-4, 4 <= j < nxx-4
        const float* vb = a.vel + (size_t)sl.s * a.vel_stride;
        for (int k = 0; k < passes; ++k) {
            int c0 = 0, gz = 0;
            const bool valid = item_of(sc, tid, k, &c0, &gz);
            // item position: bit 31 no item, bit 30 an injection point inside, c0 << 16 | gz
            bool src_here = false;
            for (int q = 0; q < src.n && q < kMaxSrc; ++q)
                src_here |= src.lc[q] >= c0 && src.lc[q] < c0 + 4 && src.z[q] >= gz && src.z[q] < gz + 4;
            s_pos[k * kRC + tid] = (valid ? 0 : (int)0x80000000) | (valid && src_here ? 0x40000000 : 0) | (c0 << 16) | gz;
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
                    kr[8 * m + e] = __float_as_uint(ok ? -st::el(k4, e) : 0.0f);
                    kr[8 * m + 4 + e] = __float_as_uint(ok ? st::damp(rows, col, e) : 0.0f);
                }
            }
            __syncwarp();
            tmem_st32(tbase + kItemCols * k, kr);
        }
        tmem_wait_st();
    }
    __syncthreads();

    ulonglong2* stage = reinterpret_cast<ulonglong2*>(smem + 2 * (size_t)(a.wmax + 8) * lds);
    // the halo of the next level is fetched during the last two passes
    const int fetch_at = passes >= 2 ? passes - 2 : 0;
    // the drill's stalled slab publishes into the spare area after both parity slots
    const bool stalled = DRILL && (int)blockIdx.x == a.stall;
    const size_t mstep = stalled ? 1 : (size_t)a.nslab, mbase = stalled ? 2 * (size_t)a.nslab : blockIdx.x;
    const uint32_t limit = DRILL ? a.spin : tma::kSpinLimit;
    bool done = !fits;
    for (int t = a.t_begin; t < a.t_end && !done; ++t) {
        float* A = smem + oa;  // Q^t (stencil)
        float* B = smem + ob;  // Q^{t-1}, then Q^{t+1}
        // level L computes Q^{t+1} and publishes its edges with tag L + 1,
        // which the neighbours fetch into their halo during this same level
        const unsigned lv = (unsigned)(t - a.t_begin);
        const unsigned tag = lv + 1;
        const size_t slot = tag & 1u;
        const bool fetch = t + 1 < a.t_end;
        if (a.seis && t > a.tlag) {
#pragma unroll
            for (int j = 0; j < kRecPerThread; ++j)
                if (rec_idx[j] >= 0) a.seis[rec_off[j] + (t - a.tlag)] = rec_d[j] * A[rec_idx[j]];
        }
        const int sample = (t + 1 < a.nt) ? t + 1 : -1;
        ulonglong2* mine = a.xbuf + (DRILL ? slot * mstep + mbase : slot * a.nslab + blockIdx.x) * 2 * nw;
        const ulonglong2* from_left = a.xbuf + (slot * a.nslab + (sl.left >= 0 ? sl.left : 0)) * 2 * nw + nw;
        const ulonglong2* from_right = a.xbuf + (slot * a.nslab + (sl.right >= 0 ? sl.right : 0)) * 2 * nw;
        for (int k = 0; k <= passes; ++k) {
            if (k == fetch_at && fetch) {
#pragma unroll
                for (int i = 0; i < kMaxXW; ++i) {
                    const int w = tid + i * kRT;
                    if (xdst[i] >= 0) cp_async16(stage + w, w < nw ? from_left + w : from_right + (w - nw));
                }
            }
            if (k == passes) break;
            const int pos = s_pos[k * kRC + tid];
            const bool valid = pos >= 0;
            const int c0 = (pos >> 16) & 0x3fff, gz = pos & 0xffff;
            ulonglong2* pa = (sl.left >= 0 && c0 == 0) ? mine : nullptr;  // the edge runs
            ulonglong2* pb = (sl.right >= 0 && c0 + 4 >= sl.w) ? mine + nw : nullptr;
            res_item(a, A, B, lds, c0, gz, valid, (pos & 0x40000000) != 0, tbase + kItemCols * k, src, sample, pa, pb,
                     tag);
        }
        if (fetch) {
            // unpack the words this thread fetched into the halo of B (Q^{t+1});
            // a word not yet at this level is polled from L2 (bounded)
            cp_async_wait_all();
            bool ok = true;
#pragma unroll
            for (int i = 0; i < kMaxXW; ++i) {
                const int w = tid + i * kRT;
                if (xdst[i] < 0) continue;
                ulonglong2 v = stage[w];
                if (!word_is(v, tag)) {
                    const ulonglong2* g = w < nw ? from_left + w : from_right + (w - nw);
                    uint32_t spin = 0;
                    for (; spin < limit; ++spin) {
                        v = ld_word(g);
                        if (word_is(v, tag)) break;
                        if (DRILL && (spin & 31u) == 31u && tma::ld_flag(a.err)) {
                            spin = limit;  // another slab has failed: give up now
                            break;
                        }
                        __nanosleep(64);
                    }
                    ok = ok && spin < limit;
                }
                *reinterpret_cast<float2*>(B + xdst[i]) =
                    make_float2(__uint_as_float((unsigned)v.x), __uint_as_float((unsigned)v.y));
            }
            if (!ok) {
                atomicExch(a.err, 1);
                abort_flag = 1;
            }
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

// column pitches (ldz + 8) compiled as constants: ldz a multiple of 32 up to 384
#define FWI_FWD_RES_LDS(X) X(40) X(72) X(104) X(136) X(168) X(200) X(232) X(264) X(296) X(328) X(360) X(392)

const void* res_kernel(int ldz, bool drill) {
    if (drill) return (const void*)fwd_res_kernel<0, true>;
#define FWI_X(l) if (ldz + 8 == l) return (const void*)fwd_res_kernel<l, false>;
    FWI_FWD_RES_LDS(FWI_X)
#undef FWI_X
    return (const void*)fwd_res_kernel<0, false>;
}

bool is_drill(const FwdResArgs& a) { return a.stall >= 0 || a.spin != tma::kSpinLimit; }

cudaError_t res_configure(int ldz, size_t smem, int* ctas) {
    smem = smem < kMinSmem ? kMinSmem : smem;
    const void* fn = res_kernel(ldz, false);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(res_kernel(ldz, true), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, kRT, smem);
    return e;
}

cudaError_t res_launch(const FwdResArgs& a, size_t smem, cudaStream_t st) {
    smem = smem < kMinSmem ? kMinSmem : smem;
    void* args[] = {const_cast<FwdResArgs*>(&a)};
    return cudaLaunchCooperativeKernel(res_kernel(a.ldz, is_drill(a)), dim3(a.nslab), dim3(kRT), args, smem, st);
}

}  // namespace

int fwd_res_threads() { return kRC; }
int fwd_res_max_rec() { return kRecPerThread * kRC; }
int fwd_res_max_src() { return kMaxSrc; }
bool fwd_res_fits(int w, int ldz) {
    const Sched sc = make_sched(w, ldz);
    return sc.passes <= kMaxPasses && 4 * ldz <= kMaxXW * kRT;
}

size_t fwd_res_stage_smem(int ldz) { return (size_t)4 * ldz * sizeof(ulonglong2); }

size_t fwd_res_smem(int wmax, int ldz) {
    // two field buffers of (wmax + 8) columns, then the staging of 4 ldz halo words
    const size_t need = (size_t)2 * (wmax + 8) * (ldz + 8) * sizeof(float) + fwd_res_stage_smem(ldz);
    return need < kMinSmem ? kMinSmem : need;
}

size_t fwd_res_static_smem() {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fwd_res_kernel<0, false>) != cudaSuccess) {
        cudaGetLastError();
        return sizeof(SrcList) + 64;
    }
    return fa.sharedSizeBytes;
}

cudaError_t fwd_res_configure(int ldz, size_t smem, int* ctas_per_sm) { return res_configure(ldz, smem, ctas_per_sm); }

cudaError_t launch_fwd_res(const FwdResArgs& a, size_t smem, cudaStream_t st) { return res_launch(a, smem, st); }

}  // namespace fwi
