// engine.hpp — device state and workflows behind the C ABI (fwi2d.h).
//
// One Engine per context.  It owns one CUDA stream, the survey-sized device
// buffers (seismograms, data, residuals), the per-batch wavefields and the
// CUDA graphs of the time loops.  Shots are processed in batches: every step
// of a batch is one launch over all of its shots (blockIdx.z = shot), and the
// whole nt+tlag step loop is captured once per (propagation kind, batch size)
// as a CUDA graph and replayed for every batch.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/fwi2d.h"
#include "host.hpp"
#include "kargs.h"
#include "kernels.h"

namespace fwi {

class Engine {
public:
    Engine(const std::string& params_path, int mode);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    fwi_dims dims() const;
    cudaStream_t stream() const { return st_; }
    void stream_sync() { sync("stream"); }
    // restarts the sequence of random boundaries (one per gradient pass)
    void set_seed(uint64_t s) {
        seed_ = s;
        rbc_epoch_ = 0;
    }
    long long launches(bool reset) { long long c = launches_; if (reset) launches_ = 0; return c; }
    // forward-kernel timing (events around each forward propagation launch)
    void fwd_timing(bool enable);
    void fwd_timing_read(double* ms, long long* launches, long long* updates);
    void bwd_timing_read(double* ms, long long* launches, long long* updates);

    void set_model(const float* vp_host);          // nz x nx
    void get_model(float* vp_host);
    void get_wavelet(float* w) const;
    void get_indices(int shot, int* src_xz, int* rec_x, int* rec_z) const;
    // aperture window of a shot: model columns [c0, c0 + w)
    void get_window(int shot, int* c0, int* w) const;

    // modeling
    void model_shots(int s0, int ns, float* seis_out, bool out_on_device);
    // migration
    void rtm_reset();
    void rtm_shots(int s0, int ns, const float* data, bool data_on_device);
    void rtm_image(float* image_host);
    void rtm_raw(float* img_host, float* illum_host);
    // inversion
    void set_observed(const float* obs, bool on_device);
    double compute_gradient(bool with_gradient);
    // sharded inversion: compute_gradient = accumulate_gradient (shots of the
    // range, raw accumulators) + finish_gradient (post-processing)
    void set_shot_range(int s0, int ns);
    int range_s0() const { return range_s0_; }
    int range_n() const { return range_n_; }
    // float offset of shot s's seismogram in an all-shots buffer
    size_t survey_offset(int s) const { return (size_t)s * nrec_ * nt_; }
    double accumulate_gradient(bool with_gradient);
    void finish_gradient();
    void accumulators(float** a, float** b) const;
    void trial_steps(float* a1, float* a2) const;
    float parabola_step(float f0, float f1, float f2) const;
    void get_gradient(float* g_host);
    // replaces the search direction of the line search / update (normalised
    // by its max |d| like the gradient): d_dir or host dir, nz x nx
    void set_direction(const float* dir, bool on_device);
    float* direction_dev() const { return d_grad_; }
    void get_gradient_raw(float* g_host, float* illum_host);
    double linesearch_trial(float alpha);
    float optimization(float f0);
    void update_model(float step, float* vp_out, float vmin = 0.0f, float vmax = 0.0f);
    // data preparation (run/generate_input_data.py:22-44, run/generate_setup.py:49-51)
    void mute_direct(float* data_all, bool on_device, float velocity, float delay, float gstd);
    void smooth_model(const float* vp_host, float sigma, float depth_mask, float* out_host);
    // random boundary of one shot on the RBC grid, nzz x nxx unpitched
    void random_boundary(int shot, float* out_host);

    // accessors used by the executables
    const ParamFile& params() const { return P_; }
    const Geometry& geometry() const { return geo_; }
    int nx() const { return nx_; }
    int nz() const { return nz_; }
    int nt() const { return nt_; }
    float dh() const { return dh_; }
    float dt() const { return dt_; }
    float fmax() const { return fmax_; }
    int max_iteration() const { return max_iteration_; }

private:
    struct Grid {
        int nb = 0;
        int nxx = 0;       // widest shot grid (window + 2 nb); every shot's when not windowed
        int nzz = 0, ldz = 0;
        int full_nxx = 0;  // nx + 2 nb: the padded whole model
        long long fstride() const { return (long long)ldz * nxx; }
    };
    // Per-grid shot tables (indices depend on nb).
    struct Tables {
        std::vector<ShotDesc> shots;       // one per survey shot
        std::vector<int> src_x, src_z;     // grid indices on the padded whole model
        std::vector<int> rec_x, rec_z;     // per receiver (same for all shots)
        std::vector<int> nxx;              // per shot: width of its grid
        int* d_rec_pt = nullptr;           // nsrc*nrec
        int* d_src_colptr = nullptr;       // nsrc*(nxx+1)
        int* d_src_z = nullptr;
        long long* d_src_soff = nullptr;
        int* d_rec_colptr = nullptr;       // nsrc*(nxx+1)
        int* d_rec_z = nullptr;            // nsrc*nrec, sorted by column
        long long* d_rec_soff = nullptr;
        std::vector<int> h_src_colptr, h_rec_colptr;  // host copies of the column tables
        std::vector<int> h_rec_ent_z;                  // host copies of the receiver entries' rows
        std::vector<long long> h_rec_ent_soff;         // and trace offsets (indexed like d_rec_z)
    };
    enum Kind { kFwdRecord = 0, kFwdNoRecord = 1, kBwdImage = 2, kBwdGradient = 3 };

    void setup_grid(Grid* g, Tables* t, int nb);
    void free_tables(Tables* t);
    void alloc_buffers();
    void upload_batch(const Tables& t, int s0, int ns);
    void setup_windows();
    // velocity of the batch's shots on the RBC grid: the shared padded model,
    // or (windowed) every shot's window padded by edge replication
    void rbc_base(int s0, int ns, const float** base, long long* stride);
    void expand_to(const Grid& g, const float* d_model_interior, float* d_out);
    void build_rbc(int s0, int ns);
    // forward propagation of the current batch (fields end in fld_[0..1])
    void run_forward(const Grid& g, const Tables& t, int ns, const float* vel, long long vel_stride, bool abc,
                     bool record, float* d_seis);
    void run_backward(const Grid& g, const Tables& t, int ns, const float* vel, long long vel_stride,
                      bool gradient, const float* d_series);
    // forward-kernel choice for (grid, batch size, ABC): the simple tiled kernel
    // (k_stencil.cu) or a persistent TMA variant (k_fwd_tma.cu), autotuned
    struct FwdPlan {
        int kind = 0;                 // 0 simple, 1 TMA (per-launch), 2 multi-level, 3 resident
        FwdTmaConfig cfg{1, 32, 2};
        FwdTmaConfig tail{1, 32, 2};  // T = 1 variant for an odd last step
        int grid = 0, tail_grid = 0;
        int minb = 2;                 // multi-level kernel: CTAs per SM of its register budget
        int ipt = 0, wmax = 0;        // resident kernel: items per thread, widest slab
        size_t smem = 0;              // resident kernel: dynamic shared memory
        std::vector<ResSlab> slabs;   // resident kernel: one per CTA
        double us_per_step = 0;
        std::string tuning;           // autotuner timings of all candidates
    };
    FwdPlan fwd_plan(const Grid& g, const Tables& t, int ns, bool abc, const float* vel, long long vel_stride);
    const CUtensorMap& tmap(const float* base, const Grid& g, int nshots, int boxz, int boxx,
                            bool whole_model = false);
    void upload_tile_base(const Grid& g, int ns, int tx);
    void launch_fwd_tma_step(const FwdPlan& p, bool two, const Grid& g, const Tables& t, int ns, const float* vel,
                             long long vel_stride, bool abc, float* cur, float* old, float* out1, float* out2, int tt,
                             bool record, float* d_seis);
    double time_fwd_candidate(const FwdPlan& p, const Grid& g, const Tables& t, int ns, const float* vel,
                              long long vel_stride, bool abc);
    // backward-kernel choice: the one-level kernel of k_stencil.cu (kind 0) or
    // a cooperative multi-level variant of k_bwd_loop.cu (kind 2), autotuned
    struct BwdPlan {
        int kind = 0;
        int TX = 16, S = 3, grid = 0;
        double us_per_step = 0;
        std::string tuning;
    };
    BwdPlan bwd_plan(const Grid& g, const Tables& t, int ns, const float* vel, long long vel_stride, bool gradient,
                     const float* d_series, float* scratch0, float* scratch1);
    void launch_bwd_loop_levels(const BwdPlan& p, const Grid& g, const Tables& t, int ns, const float* vel,
                                long long vel_stride, bool gradient, const float* d_series, float* const ps[2],
                                float* const pr[2], int b_begin, int b_end, long long timed_updates = -1);
    void launch_fwd_loop_levels(const FwdPlan& p, const Grid& g, const Tables& t, int ns, const float* vel,
                                long long vel_stride, bool abc, bool record, float* d_seis, int t_begin, int t_end,
                                long long timed_updates = -1);
    // shared-memory-resident forward kernel (k_fwd_res.cu): slabs of the batch
    // when its two time levels fit the SMs' shared memory
    bool plan_resident(const Grid& g, const Tables& t, int ns, FwdPlan* p);
    void launch_fwd_res_levels(const FwdPlan& p, const Grid& g, const Tables& t, const float* vel,
                               long long vel_stride, bool abc, float* d_seis, const float* in_cur,
                               const float* in_old, float* out_cur, float* out_old, int t_begin, int t_end,
                               long long timed_updates = -1);
    // events of one timed forward region: begin is recorded before the
    // region's kernel(s), end after them
    struct TimedRegion {
        cudaEvent_t begin = nullptr, end = nullptr;
        long long launches = 0, updates = 0;
    };
    cudaEvent_t timing_event();
    void timing_begin(TimedRegion* r);
    void timing_end(TimedRegion* r, long long launches, long long updates);
    void check(cudaError_t e, const char* what);
    void sync(const char* what);
    void check_finite(const float* d, size_t n, const char* what);
    int h_shot_nxx(const Grid& g, int s /*batch-local shot*/) const {
        return batch_t_ ? batch_t_->nxx[batch_s0_ + s] : g.nxx;
    }
    // padded grid points of a batch of ns shots (one time level)
    long long batch_points(const Grid& g, int ns) const {
        long long n = 0;
        for (int s = 0; s < ns; ++s) n += (long long)g.nzz * h_shot_nxx(g, s);
        return n;
    }
    void ensure_rbc_base();
    double residual_of(int s0, int ns, const float* d_obs, const float* d_cal, float* d_res);

    ParamFile P_;
    int mode_;
    Geometry geo_;
    int nx_ = 0, nz_ = 0, nt_ = 0, tlag_ = 0, nsrc_ = 0, nrec_ = 0;
    float dh_ = 0, dt_ = 0, fmax_ = 0, idh2_ = 0;
    float vmin_ = 0, vmax_ = 0;
    std::vector<float> wavelet_, b1d_;
    Grid abc_, rbc_;
    Tables abc_t_, rbc_t_;
    bool has_abc_ = false, has_rbc_ = false;
    float rbc_ratio_ = 0, rbc_varVp_ = 0;
    float zmask_ = 0;
    int max_iteration_ = 0;
    uint64_t seed_ = 0;
    long long rbc_epoch_ = 0;
    int batch_ = 1;
    long long launches_ = 0;
    int range_s0_ = 0, range_n_ = 0;    // shots of compute_gradient / linesearch_trial
    // aperture windows
    std::vector<Window> win_;
    bool windowed_ = false;
    int* d_full_win_ = nullptr;          // {0} and {nx}: the whole-model window
    float* d_geo_ = nullptr;             // sx, sz (nsrc each), rx, rz (nrec each)
    unsigned* d_shot_bits_ = nullptr;    // nsrc scratch words
    double* d_weights_ = nullptr;        // Gaussian half-kernel (up to 1024 taps)
    unsigned char* d_trace_keep_ = nullptr;  // per trace: receiver inside the shot's window
    // batch being propagated (tables and first survey shot)
    const Tables* batch_t_ = nullptr;
    int batch_s0_ = 0;

    cudaStream_t st_ = nullptr;
    // model state
    float* d_vp_ = nullptr;          // interior velocity nz x nx
    float* d_m_ = nullptr;           // slowness^2 (inversion)
    float* d_vel_abc_ = nullptr;     // padded ABC-grid velocity (shared by shots)
    float* d_vel_rbc_base_ = nullptr;// padded RBC-grid edge-replicated velocity
    bool vel_abc_valid_ = false, vel_rbc_valid_ = false;
    float* d_wavelet_ = nullptr;
    float* d_b1d_ = nullptr;
    // batch state
    ShotDesc* d_batch_ = nullptr;    // device copy of the batch's shot descriptors
    ShotDesc* h_batch_ = nullptr;    // pinned staging
    int* d_batch_nxx_ = nullptr;     // per batch shot: width (RBC kernel)
    int* d_batch_id_ = nullptr;      // per batch shot: survey index
    int* d_batch_c0_ = nullptr;      // per batch shot: window start column
    int* d_batch_w_ = nullptr;       // per batch shot: window width
    int* d_bump_ptr_ = nullptr;
    BumpDev* d_bumps_ = nullptr;
    size_t bumps_cap_ = 0;
    // multi-level backward kernel: receiver points per CTA (built per launch)
    int* d_inj_ptr_ = nullptr;
    InjPoint* d_inj_pts_ = nullptr;
    long long* d_inj_soff_ = nullptr;
    size_t inj_ptr_cap_ = 0, inj_pts_cap_ = 0, inj_soff_cap_ = 0;
    std::vector<int> h_inj_ptr_;
    std::vector<InjPoint> h_inj_pts_;
    std::vector<long long> h_inj_soff_;
    void upload_injection_points(const Grid& g, const Tables& t, int ns, int tx, int grid);
    // multi-level forward kernel: receiver entries per CTA (built per launch)
    int* d_rec_ptr_ = nullptr;
    RecPoint* d_rec_pts_ = nullptr;
    size_t rec_ptr_cap_ = 0, rec_pts_cap_ = 0;
    std::vector<int> h_rec_ptr_;
    std::vector<RecPoint> h_rec_pts_;
    void upload_record_points(const Grid& g, const Tables& t, int ns, int tx, int grid);
    float* fld_[4] = {nullptr, nullptr, nullptr, nullptr};
    float* acc_[2] = {nullptr, nullptr};
    float* d_vel_batch_ = nullptr;   // per-shot RBC velocity
    long long fstride_max_ = 0;
    // survey buffers
    float* d_seis_ = nullptr;        // modeled / calculated data, nsrc*nrec*nt
    float* d_data_ = nullptr;        // observed (inversion) or input (migration) data
    float* d_res_ = nullptr;         // residual / adjoint source
    double* d_partial_ = nullptr;
    double* d_sum_ = nullptr;
    int* d_flag_ = nullptr;
    unsigned int* d_gmax_ = nullptr;
    // cropped accumulators nz x nx
    float* d_img_ = nullptr;
    float* d_illum_ = nullptr;
    float* d_grad_ = nullptr;        // post-processed gradient
    float* d_tmp_ = nullptr;
    bool have_obs_ = false, have_grad_ = false;
    // time-loop graphs, key = (kind, grid, batch size)
    std::map<long long, cudaGraphExec_t> graphs_;
    bool use_graphs_ = true;
    // TMA forward path
    std::map<std::string, CUtensorMap> tmaps_;
    std::map<long long, FwdPlan> plans_;
    std::map<long long, BwdPlan> bwd_plans_;
    std::string bwd_kernel_ = "auto";  // key bwd_kernel: auto | simple | loop:TX,S
    int* d_tile_base_ = nullptr;
    int* d_err_ = nullptr;
    unsigned* d_sync_ = nullptr;       // grid-barrier counter of the multi-level kernel
    ResSlab* d_slabs_ = nullptr;       // resident kernel: slab table and halo exchange words
    ulonglong2* d_xbuf_ = nullptr;
    size_t slabs_cap_ = 0, xbuf_cap_ = 0;
    int sm_count_ = 0;
    // bounded device waits: polls before a wait gives up (key test_wait_limit,
    // default 2^22); failure drill (keys test_stall_fwd / test_stall_bwd): the
    // CTA of that index in the multi-level / resident forward or the
    // multi-level backward kernel withholds its work so the others' waits run
    // out (-1: off)
    unsigned spin_limit_ = 1u << 22;
    int stall_fwd_ = -1, stall_bwd_ = -1;
    std::string fwd_kernel_ = "auto";  // key fwd_kernel: auto | simple | tma:T,TX,S
    float* fwd_cur_ = nullptr;         // Q^N after run_forward
    float* fwd_old_ = nullptr;         // Q^{N-1}
    // forward-kernel timing
    bool timing_ = false;
    std::vector<TimedRegion> timed_;
    std::vector<cudaEvent_t> event_pool_;
    double timed_ms_ = 0;
    long long timed_launches_ = 0, timed_updates_ = 0;
    // the same for the backward kernel (TimedRegion.launches < 0 marks them)
    double btimed_ms_ = 0;
    long long btimed_launches_ = 0, btimed_updates_ = 0;
public:
    // plan used by the last forward propagation (for reporting)
    std::string last_fwd_plan;
    std::string last_bwd_plan;
};

}  // namespace fwi
