/*
 * fwi2d.h — C ABI of the B200 wave-propagation engine (libfwi2d.so).
 *
 * The reference (phbastosa/FWI2D) has no library interface: its boundary is the
 * three executables and the C++ classes they drive
 *   Modeling   src/modeling/modeling.cuh:18-87
 *   Migration  src/migration/migration.cuh:6-38
 *   Inversion  src/inversion/inversion.cuh:6-83
 * Each entry point below replaces one of those class methods (cited per
 * function) so that the drop-in executables, the Python mirror and any foreign
 * caller (ctypes, cgo, JNI) bind the same plain-C surface.
 *
 * Conventions
 *   - Every function returns an int status: FWI_OK (0) or a negative FWI_ERR_*.
 *     The message of the last failure is fwi_last_error(ctx) (ctx may be NULL
 *     for failures of fwi_ctx_create).
 *   - Host arrays are caller-owned and use the reference's file layouts:
 *       model / image / gradient : nz x nx float32, z fastest (idx = i + j*nz)
 *       seismogram of one shot   : nt x nrec float32, trace-major (t + r*nt)
 *       all shots                : nsrc consecutive seismograms
 *   - "_dev" variants take device pointers (same layouts) and leave data in HBM.
 *   - Device memory is owned by the context; one CUDA stream per context; a
 *     context is not thread-safe.  Functions write nothing to stdout.
 */
#ifndef FWI2D_H
#define FWI2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define FWI_OK            0
#define FWI_ERR_PARAM    -1   /* missing / malformed parameters.txt key      */
#define FWI_ERR_IO       -2   /* file open / short read / write failure       */
#define FWI_ERR_CUDA     -3   /* CUDA runtime error                           */
#define FWI_ERR_CFL      -4   /* vmax*dt/dh above the 8th-order 2-D limit     */
#define FWI_ERR_NAN      -5   /* non-finite wavefield, seismogram or misfit   */
#define FWI_ERR_TIMEOUT  -6   /* a bounded device wait gave up                */
#define FWI_ERR_STATE    -7   /* call out of order (e.g. gradient before data)*/
#define FWI_ERR_ARG      -8   /* bad argument (NULL, shot out of range, size) */
#define FWI_ERR_NOMEM    -9   /* device allocation failed                     */

/* ---- workflow a context is created for ---------------------------------- */
#define FWI_MODE_MODELING  0  /* ABC boundary, keys of modeling.cu:17-30,113-150 */
#define FWI_MODE_MIGRATION 1  /* RBC boundary, keys of migration.cu:3-36          */
#define FWI_MODE_INVERSION 2  /* ABC + RBC grids, keys of inversion.cu:3-53       */

typedef struct fwi_ctx fwi_ctx;

typedef struct fwi_dims {
    int   nx, nz;          /* model samples                                  */
    int   nt;              /* time samples                                   */
    int   nsrc, nrec;      /* shots, receivers (from SPS / RPS)              */
    int   nb;              /* boundary cells of the primary grid             */
    int   nxx, nzz;        /* padded primary grid (nx+2nb, nz+2nb)           */
    int   ldz;             /* device column pitch (floats, multiple of 32)   */
    int   tlag;            /* wavelet delay in samples, int(t0/dt)+1         */
    int   abc_nb, rbc_nb;  /* inversion: the two boundary widths             */
    float dh, dt, fmax;
    float vmin, vmax;      /* of the model given at creation                 */
} fwi_dims;

/* ---- context -------------------------------------------------------------
 * Replaces Modeling::set_parameters (modeling.cu:3-15), Migration::set_parameters
 * (migration.cu:3-36) and Inversion::set_parameters (inversion.cu:3-53): parses
 * params_path with the reference's key rules (admin.cpp:53-98), reads SPS/RPS
 * (geometry.cpp:3-43) and model_file, builds the wavelet (modeling.cu:32-90)
 * and damping tables (modeling.cu:113-150) and allocates device state. */
int  fwi_ctx_create(const char* params_path, int mode, fwi_ctx** ctx);
void fwi_ctx_destroy(fwi_ctx* ctx);
const char* fwi_last_error(const fwi_ctx* ctx);
int  fwi_get_dims(const fwi_ctx* ctx, fwi_dims* out);
/* The context's CUDA stream (cudaStream_t) for callers that time or order work. */
int  fwi_get_stream(const fwi_ctx* ctx, void** stream);
/* Value of a parameters.txt key under the reference's rules (admin.cpp:53-98);
 * FWI_ERR_PARAM when absent, FWI_ERR_ARG when buf (len bytes) is too small. */
int  fwi_get_param(const fwi_ctx* ctx, const char* key, char* buf, size_t len);
/* Seed of the random-boundary generator (default from key rbc_seed, else 0);
 * restarts the sequence of per-gradient-pass boundaries. */
int  fwi_set_seed(fwi_ctx* ctx, uint64_t seed);

/* Velocity model, nz x nx.  Replaces set_properties/expand_boundary
 * (modeling.cu:152-218) for a model already in memory. */
int  fwi_set_model(fwi_ctx* ctx, const float* vp);
int  fwi_get_model(fwi_ctx* ctx, float* vp);
/* Wavelet actually injected (nt floats, before the idh2 scale). */
int  fwi_get_wavelet(fwi_ctx* ctx, float* w);
/* Grid indices of shot `shot`: sIdx,sIdz (2 ints) and rIdx[nrec], rIdz[nrec];
 * initialization, modeling.cu:252-277.  Any pointer may be NULL. */
int  fwi_get_indices(fwi_ctx* ctx, int shot, int* src_xz, int* rec_x, int* rec_z);
/* Aperture window of shot `shot`: model columns [*c0, *c0 + *w).  The whole
 * model (0, nx) unless the parameter file sets aperture_offset (maximum
 * offset in metres, every shot) or aperture_file (a text file with one maximum
 * offset per shot).  A windowed shot is modeled on its
 * window padded by the boundary; receivers outside it record nothing and, in
 * an inversion, their traces take no part in the misfit.  No reference
 * counterpart: the reference models every shot on the whole model. */
int  fwi_get_window(fwi_ctx* ctx, int shot, int* c0, int* w);

/* ---- modeling ------------------------------------------------------------
 * One shot: initialization + forward_solver + get_seismogram without the file
 * write (modeling.cu:252-299, 347-353). */
int  fwi_model_shot(fwi_ctx* ctx, int shot, float* seis);
/* All shots, batched on the device: seis_all holds nsrc seismograms. */
int  fwi_model_survey(fwi_ctx* ctx, float* seis_all);
int  fwi_model_survey_dev(fwi_ctx* ctx, float* d_seis_all);

/* ---- reverse-time migration ---------------------------------------------
 * Migration::forward_propagation + backward_propagation for one shot, or all
 * shots batched (migration.cu:49-81, 117-180).  data is the shot's input
 * seismogram (nt x nrec); image and illumination accumulate in the context
 * until fwi_rtm_reset. */
int  fwi_rtm_reset(fwi_ctx* ctx);
int  fwi_rtm_shot(fwi_ctx* ctx, int shot, const float* data);
int  fwi_rtm_survey(fwi_ctx* ctx, const float* data_all);
int  fwi_rtm_survey_dev(fwi_ctx* ctx, const float* d_data_all);
/* Migration::export_seismic without the file write (migration.cu:90-115):
 * crop, image/illumination, -d2/dz2. */
int  fwi_rtm_image(fwi_ctx* ctx, float* image);
/* Raw accumulators (nz x nx, cropped): cross-correlation and illumination. */
int  fwi_rtm_raw(fwi_ctx* ctx, float* image, float* illum);

/* ---- full-waveform inversion --------------------------------------------
 * Observed data of all shots (nsrc x nt x nrec), kept on the device for the
 * gradient and line-search modelings (set_obs_data, inversion.cu:168-172). */
int  fwi_set_observed(fwi_ctx* ctx, const float* obs_all);
int  fwi_set_observed_dev(fwi_ctx* ctx, const float* d_obs_all);
/* Inversion::compute_gradient (inversion.cu:111-166): ABC modeling, residual,
 * FP64 misfit, and - when with_gradient != 0 - RBC forward + adjoint back-
 * propagation + gradient post-processing.  *sum_res = sum of residual^2.
 * A non-finite misfit (a model made unstable by an unbounded update) returns
 * FWI_ERR_NAN where the reference would carry NaN on. */
int  fwi_compute_gradient(fwi_ctx* ctx, int with_gradient, double* sum_res);
/* ---- sharded inversion (shots split over processes / GPUs) ---------------
 * fwi_compute_gradient(ctx, 1, s) equals fwi_gradient_accumulate followed by
 * fwi_gradient_finish.  A process that owns shots [s0, s0+ns) sets its range,
 * accumulates, sums the two raw accumulators (and the misfit) over all
 * processes in place - e.g. an NCCL all-reduce on the device buffers that
 * fwi_accumulators returns - and then finishes; fwi_linesearch_trial sums over
 * the range too, and fwi_parabola_step turns the summed misfits into the step
 * of optimization (inversion.cu:286-308).  The range (default: all shots)
 * applies to fwi_compute_gradient, fwi_gradient_accumulate and
 * fwi_linesearch_trial. */
int  fwi_set_shot_range(fwi_ctx* ctx, int s0, int ns);
int  fwi_gradient_accumulate(fwi_ctx* ctx, int with_gradient, double* sum_res);
int  fwi_gradient_finish(fwi_ctx* ctx);
/* Device pointers (nz x nx floats each, owned by the context) of the raw
 * cross-correlation (RTM image or FWI gradient) and source-illumination
 * accumulators; the context's stream is idle when the call returns. */
int  fwi_accumulators(fwi_ctx* ctx, float** d_image_or_gradient, float** d_illum);
/* Trial steps a1 = 0.02 dm, a2 = 0.05 dm of the current model and the
 * parabola vertex of misfits f0, f1, f2 at 0, a1, a2 (inversion.cu:286-308). */
int  fwi_trial_steps(fwi_ctx* ctx, float* a1, float* a2);
int  fwi_parabola_step(fwi_ctx* ctx, float f0, float f1, float f2, float* step);
/* Replaces the search direction of fwi_linesearch_trial / fwi_optimization /
 * fwi_update_model (m -= step * d) by dir (nz x nx, slowness^2 units),
 * normalised by its max |d| as the gradient is: a preconditioned direction,
 * e.g. the CNN's.  _dev: dir is a device pointer. */
int  fwi_set_direction(fwi_ctx* ctx, const float* dir);
int  fwi_set_direction_dev(fwi_ctx* ctx, const float* d_dir);
/* Post-processed gradient (nz x nx, normalised by max |g|) */
int  fwi_get_gradient(fwi_ctx* ctx, float* g);
/* Raw gradient and illumination (nz x nx, cropped, before post-processing). */
int  fwi_get_gradient_raw(fwi_ctx* ctx, float* g, float* illum);
/* Inversion::linesearch (inversion.cu:310-342): models all shots at slowness^2
 * m - alpha*g and returns the FP64 sum of residual^2. */
int  fwi_linesearch_trial(fwi_ctx* ctx, float alpha, double* sum_res);
/* Inversion::optimization (inversion.cu:286-308): the parabola through
 * (0,f0), (a1,f1), (a2,f2) with a1,a2 = 0.02,0.05*(1/vmin^2-1/vmax^2). */
int  fwi_optimization(fwi_ctx* ctx, float f0, float* step);
/* Inversion::update_model (inversion.cu:344-358) without the file write:
 * m -= step*g; velocity = 1/sqrt(m).  vp_out (nz x nx) may be NULL. */
int  fwi_update_model(fwi_ctx* ctx, float step, float* vp_out);
/* The same with the new velocity kept inside [vmin, vmax] (no reference
 * counterpart: the reference's update has no safeguard). */
int  fwi_update_model_bounded(fwi_ctx* ctx, float step, float vmin, float vmax, float* vp_out);

/* ---- data preparation ----------------------------------------------------
 * The reference prepares RTM input and the FWI starting model in Python;
 * these run the same arithmetic on the GPU.
 * fwi_mute_direct: run/generate_input_data.py:22-44 on all shots of data_all
 * (nsrc x nt x nrec, in place): each shot divided by its max |amplitude|,
 * samples t < tId[r] = int((dist_r / velocity + delay) / dt) of trace r
 * tapered by exp(-0.5 ((t - tId[r]) / gstd)^2), dist_r the source-receiver
 * distance from SPS/RPS.  The script's constants: velocity 3600, delay 0.18,
 * gstd 30 (samples). */
int  fwi_mute_direct(fwi_ctx* ctx, float* data_all, float velocity, float delay, float gstd);
int  fwi_mute_direct_dev(fwi_ctx* ctx, float* d_data_all, float velocity, float delay, float gstd);
/* run/generate_setup.py:49-51: vp_out = 1 / G(1 / vp) with G the separable
 * Gaussian filter of scipy.ndimage (sigma in cells, radius int(4 sigma + 0.5),
 * mode 'reflect', z pass then x pass), rows above int(depth_mask / dh) kept
 * from vp.  nz x nx host arrays; the script uses sigma 3. */
int  fwi_smooth_model(fwi_ctx* ctx, const float* vp, float sigma, float depth_mask, float* vp_out);

/* ---- random boundary ----------------------------------------------------
 * set_random_boundary (modeling.cu:431-531) for shot `shot` of the current
 * model, on the context's RBC grid; out is nzz x (w + 2 nb) (z fastest,
 * unpitched), w the shot's window width (nx without windows). */
int  fwi_random_boundary(fwi_ctx* ctx, int shot, float* vp_rbc);

/* ---- host-side utilities (no GPU, no context) -----------------------------
 * The set-up steps of the engine, exposed for callers that prepare inputs and
 * for CPU-side checks. */
/* catch_parameter (admin.cpp:53-98) on a file. */
int  fwi_util_parameter(const char* params_path, const char* key, char* buf, size_t len);
/* set_wavelet (modeling.cu:32-90): nt samples and tlag. */
int  fwi_util_wavelet(int nt, float dt, float fmax, float* out, int* tlag);
/* set_abc_dampers b1d profile (modeling.cu:113-150). */
int  fwi_util_b1d(int nb, float abc_factor, float* out);
/* initialization's index rule int((c + dh/2)/dh) + nb (modeling.cu:257-269). */
int  fwi_util_grid_index(int n, const float* coord, float dh, int nb, int* out);
/* Aperture window of a source at x = xs (metres) for a maximum offset
 * max_offset: model columns [*c0, *c0 + *w) of an nx-column model (the rule of
 * fwi_get_window; no reference counterpart). */
int  fwi_util_window(float xs, float max_offset, int nx, float dh, int* c0, int* w);
/* Random-boundary bumps of one shot (modeling.cu:431-465): 5 floats
 * (xc, zc, r, A, sign) per bump; *count = bumps generated (may exceed cap). */
int  fwi_util_bumps(int nxx, int nzz, int nb, float dh, float ratio, float varVp, uint64_t seed,
                    uint32_t shot, float* out, int cap, int* count);
/* Standard-normal draw `ctr` of the random-boundary stream (seed, shot, stream). */
int  fwi_util_normal(uint64_t seed, uint32_t shot, uint32_t stream, uint64_t ctr, float* out);

/* ---- residual and misfit without device allocation -----------------------
 * No counterpart in the reference: it has no entry point of this kind.
 * d_res = d_obs - d_cal over n samples and *d_sum = sum(d_res^2) in FP64, for
 * callers that cannot call cudaMalloc - an application whose own pool owns
 * all device memory, code inside a stream capture, or a loop that must not
 * take cudaMalloc's implicit synchronisation.  All pointers are device memory
 * (d_sum: one double); `stream` is a cudaStream_t (NULL: default stream) and
 * the call only enqueues work.  The scratch is a 64 KiB file-scope device
 * array, so n is limited to FWI_NOALLOC_MAX_SAMPLES (FWI_ERR_ARG beyond it;
 * split larger inputs).  The first call on a device looks the array's device
 * address up (cudaGetSymbolAddress, which may load the library's device code
 * at that moment under CUDA's lazy module loading), so make it before any
 * stream capture.  The address is kept per device ordinal for the life of
 * the process: after cudaDeviceReset, or anything else that destroys the
 * device's primary context, it is stale and the entry point must not be
 * called again in that process.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.  A failed
 * call leaves its message for fwi_last_error(NULL); a call that succeeds
 * clears it. */
#define FWI_NOALLOC_MAX_SAMPLES ((size_t)8192 * 8192)
int  fwi_residual_noalloc(const float* d_obs, const float* d_cal, float* d_res, size_t n, double* d_sum,
                          void* stream);

/* ---- timing / diagnostics ----------------------------------------------- */
/* Text description of the forward-step kernel the autotuner chose for the last
 * propagation (e.g. "tma T=2 TX=16 S=2 grid=148"). */
int  fwi_describe(fwi_ctx* ctx, char* buf, size_t len);
/* Kernel launches issued by the context since creation (or the last reset). */
int  fwi_launch_count(fwi_ctx* ctx, long long* count, int reset);
/* Kernel timing.  fwi_fwd_timing(ctx, 1) resets the counters and
   brackets every later launch of the forward propagation kernel (a
   multi-level launch, or the graph of one-level launches of a batch) with
   CUDA events on the context stream; 0 turns it off.  fwi_fwd_timing_read
   waits for the recorded events and returns the summed device time in ms,
   the number of forward-kernel launches covered and the grid-point updates
   they performed (padded points x time levels x shots). */
int  fwi_fwd_timing(fwi_ctx* ctx, int enable);
int  fwi_fwd_timing_read(fwi_ctx* ctx, double* ms, long long* launches, long long* updates);
/* The same for the backward (migration / gradient) kernel, timed while
 * fwi_fwd_timing is on. */
int  fwi_bwd_timing_read(fwi_ctx* ctx, double* ms, long long* launches, long long* updates);

#ifdef __cplusplus
}
#endif
#endif /* FWI2D_H */
