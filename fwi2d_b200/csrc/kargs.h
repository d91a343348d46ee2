// kargs.h — argument blocks of the propagation kernels (host and device).
//
// Device layout of every padded grid: column-major with z fastest like the
// reference (idx = i + j*nzz, src/modeling/modeling.cu:308-309), but with the
// column pitch ldz rounded up to a multiple of 32 floats so that every column
// starts on a 128-byte boundary and float4 / TMA accesses stay aligned.  Rows
// nzz..ldz-1 hold zeros.  A batch of shots stores its fields back to back
// with a fixed per-shot stride (fstride = ldz * max columns).
#pragma once
#include <stdint.h>
#include <vector_types.h>

namespace fwi {

// Finite-difference coefficients of the reference (modeling.cuh:9-13):
// 1/560, 8/315, 1/5, 8/5, 205/72, as the decimal literals given there.
constexpr double kFDM1 = 0.001785714285;
constexpr double kFDM2 = 0.025396825396;
constexpr double kFDM3 = 0.200000000000;
constexpr double kFDM4 = 1.600000000000;
constexpr double kFDM5 = 2.847222222222;

struct ShotDesc {
    int nxx;             // padded width (columns) of this shot's grid
    int nrec;            // receivers of this shot (those inside its aperture)
    int rec_off;         // first entry of the shot in rec_pt[] / receiver tables
    int col_off;         // first entry of the shot's injection column table
    long long seis_off;  // float offset of the shot's nt x nrec trace-major block
    int vel_col;         // column of the velocity array that is column 0 of the
                         // shot's grid (aperture window over a shared velocity)
};

// Point injections into the field written by a step (the source of a forward
// propagation, the receivers of an adjoint / migration back-propagation).
// Points of column j of shot s are entries colptr[col_off+j] ..
// colptr[col_off+j+1]-1; each adds scale * series[soff + sample].
struct InjTable {
    const int* colptr;
    const int* z;
    const long long* soff;
    const float* series;
    int sample;          // sample index of this step, or -1 for no injection
    float scale;
};

struct FwdArgs {
    const ShotDesc* shots;    // batch-local shot descriptors
    const float* vel;         // velocity, padded layout
    long long vel_stride;     // per-shot stride of vel (0: shared by all shots)
    const float* cur;         // Q^t (read, stencil)
    float* nxt;               // Q^{t-1} on entry, Q^{t+1} on exit (pointwise)
    long long fstride;        // per-shot stride of cur / nxt
    int ldz, nzz, nb;
    float dt2idh2;            // dt^2 / dh^2
    const float* b1d;         // ABC damping profile (nb floats), NULL for none
    InjTable inj;
    const int* rec_pt;        // receiver points z + x*ldz, per shot at rec_off
    const long long* rec_soff;// trace offset (into seis) of each rec_pt entry
    float* seis;              // trace-major seismograms
    int rec_sample;           // sample recorded at this step, or -1
    int nt;
};

// Persistent TMA forward kernel (k_fwd_tma.cu): one or two time levels per
// launch, written out of place.
struct FwdTmaArgs {
    const ShotDesc* shots;
    const int* tile_base;     // batch-local prefix sums of tiles per shot (ns+1)
    int ns, ntz;              // shots in the batch, 128-row tiles per column
    int ldz, nzz, nb;
    long long fstride;
    int vel_shared;           // 1: one velocity for all shots (tensor map of 1 shot)
    float dt2idh2;
    const float* b1d;         // ABC profile or NULL
    InjTable inj;             // source table; sample1 / sample2 below
    int sample1, sample2;     // wavelet samples added to Q^{t+1}, Q^{t+2}; -1 none
    InjTable rec;             // receiver table (colptr, z, soff) of the batch
    float* seis;              // trace-major seismograms, NULL when not recording
    int rec_sample0, rec_sample1;  // samples recorded from Q^t and Q^{t+1}; -1 none
    float* out1;              // Q^{t+1}
    float* out2;              // Q^{t+2} (two-level launches)
    int* err;                 // raised when a bounded wait gives up
    unsigned spin;            // polls of a bounded wait before it gives up
    int stall;                // failure drill: this CTA withholds its first
                              // tile and its grid-barrier arrival (-1: none)
};

// A receiver entry recorded by the multi-level forward kernel: its point's
// offset in a batch field, its trace offset, its row and column in its shot's
// grid and that grid's width (for the damper of the absorbing boundary).
struct __align__(16) RecPoint {
    long long g;
    long long soff;
    int z, x, nxx, pad;
};

// Cooperative multi-level forward kernel (k_fwd_loop.cu): levels
// t_begin..t_end-1 in one launch, buffers rotating cur -> old, free -> cur.
struct FwdLoopArgs {
    FwdTmaArgs base;          // samples / outputs are set per level in the kernel
    int t_begin, t_end;
    int nt, tlag, record;
    int buf_cur, buf_old, buf_free;  // indices into bufs at t_begin
    float* bufs[4];
    unsigned* sync;           // grid-barrier counter, zero at launch
    // receivers, per CTA: the entries in the CTA's tiles (rec_cta_ptr[b] ..
    // rec_cta_ptr[b+1] of rec_pts), recorded at the end of each level
    const int* rec_cta_ptr;
    const RecPoint* rec_pts;
};

// Shared-memory-resident forward kernel (k_fwd_res.cu): CTA b owns slab b,
// columns [x0, x0+w) of shot s over the full depth.  left / right: the CTAs
// owning the neighbouring slabs of the same shot, -1 at the shot's edge.
struct ResSlab {
    int s, x0, w, left, right;
    int pad[3];
};

struct FwdResArgs {
    const ShotDesc* shots;
    const ResSlab* slabs;
    int nslab, wmax;          // CTAs (one per slab); widest slab
    int ldz, nzz, nb;
    long long fstride;        // per-shot stride of the field buffers
    const float* vel;         // velocity, padded layout
    long long vel_stride;     // per-shot stride of vel (0: shared by all shots)
    float dt2idh2;
    const float* b1d;         // ABC profile or NULL
    InjTable inj;             // source table (sample set per level)
    InjTable rec;             // receiver table (colptr, z, soff)
    float* seis;              // trace-major seismograms, NULL when not recording
    int t_begin, t_end, nt, tlag;
    const float* in_cur;      // Q^t at t_begin
    const float* in_old;      // Q^{t-1} at t_begin
    float* out_cur;           // Q^t at t_end
    float* out_old;           // Q^{t-1} at t_end
    ulonglong2* xbuf;         // halo words, two (value | level << 32) halves each:
                              // [2 parities][nslab][2 sides][2 ldz], zero at launch
    int* err;
    unsigned spin;            // polls of a bounded wait before it gives up
    int stall;                // failure drill: this slab publishes no halo (-1: none)
};

struct FwdTmaConfig {
    int T;    // time levels per launch (1 or 2)
    int TX;   // tile columns
    int S;    // pipeline stages
};

// Cooperative multi-level backward kernel (k_bwd_loop.cu): back-propagation
// levels b_begin..b_end-1 of a batch in one launch.  Level b reads the source
// field through the stencil from ps[(b+1)&1] and pointwise from ps[b&1] (and
// overwrites it), the receiver field through the stencil from pr[b&1] and
// pointwise from pr[(b+1)&1] (overwritten), as run_backward alternates them.
// A grid point that receives injected samples in the multi-level backward
// kernel: its offset in a batch field and its entries [e0, e1) of the
// trace-offset list (several receivers can share a point).
struct __align__(16) InjPoint {
    long long g;
    int e0, e1;
};

struct BwdLoopArgs {
    const ShotDesc* shots;
    const int* tile_base;     // prefix sums of tiles per shot (ns+1)
    int ns, ntz;
    int ldz, nzz;
    long long fstride;        // per-shot stride of fields, accumulators and velocity
    int vel_shared;           // 1: one velocity for all shots
    float dt2idh2, dt, idh2;
    InjTable inj;             // receiver-side injection table of the batch
    int nt;
    int b_begin, b_end;
    float* ps[2];
    float* pr[2];
    float* acc_a;
    float* acc_b;
    // receiver injection, per CTA: the points of the receivers in the CTA's
    // tiles (inj_cta_ptr[b] .. inj_cta_ptr[b+1] of inj_pts) and the trace
    // offsets of their entries; the series and scale are inj's
    const int* inj_cta_ptr;
    const InjPoint* inj_pts;
    const long long* inj_soff;
    int* err;
    unsigned* sync;           // grid-barrier counter, zero at launch
    unsigned spin;            // polls of a bounded wait before it gives up
    int stall;                // failure drill: this CTA withholds its first
                              // tile and its grid-barrier arrival (-1: none)
};

struct BwdArgs {
    const ShotDesc* shots;
    const float* vel;
    long long vel_stride;
    const float* ps_st;       // source field read by the stencil (Psold)
    float* ps_io;             // source field read pointwise and overwritten (Ps)
    const float* pr_st;       // receiver field read by the stencil (Pr)
    float* pr_io;             // receiver field read pointwise and overwritten (Prold)
    long long fstride;
    float* acc_a;             // image (RTM) or gradient (FWI), per shot
    float* acc_b;             // source illumination, per shot
    long long acc_stride;
    int ldz, nzz;
    float dt2idh2, dt, idh2;
    InjTable inj;             // receiver-side injection into pr_io
};

}  // namespace fwi
