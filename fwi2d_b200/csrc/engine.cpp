// engine.cpp — see engine.hpp.  Host code compiled with -ffp-contract=off.
#include "engine.hpp"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <sstream>
#include <type_traits>

namespace fwi {

namespace {
constexpr int kBufFields = 4;
// Distinct random boundaries per gradient pass: the RBC seed of pass e is
// seed + e * kEpochStride (odd constant, so passes never collide).
constexpr uint64_t kEpochStride = 0xD1B54A32D192ED03ull;
}  // namespace

void Engine::check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(FWI_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

void Engine::sync(const char* what) {
    check(cudaGetLastError(), what);
    check(cudaStreamSynchronize(st_), what);
    if (d_err_) {
        int err = 0;
        check(cudaMemcpy(&err, d_err_, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
        if (err) {
            cudaMemset(d_err_, 0, sizeof(int));
            throw Error(FWI_ERR_TIMEOUT, std::string(what) +
                                             ": a kernel gave up a bounded wait (tile loads, halo exchange) or met a "
                                             "slab its tables do not hold");
        }
    }
}

template <typename T>
static T* dalloc(size_t n, const char* what) {
    T* p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(FWI_ERR_NOMEM, std::string("cudaMalloc of ") + what + " (" + std::to_string(n * sizeof(T)) +
                                       " bytes): " + cudaGetErrorString(e));
    }
    return p;
}

static int round_up(int v, int m) { return (v + m - 1) / m * m; }

// ------------------------------------------------------------------ set-up
Engine::Engine(const std::string& params_path, int mode) : P_(params_path), mode_(mode) {
    if (mode < FWI_MODE_MODELING || mode > FWI_MODE_INVERSION) throw Error(FWI_ERR_ARG, "unknown mode");
    // set_main_parameters, modeling.cu:17-30
    nx_ = P_.i("x_samples");
    nz_ = P_.i("z_samples");
    dh_ = P_.f("model_spacing");
    nt_ = P_.i("time_samples");
    dt_ = P_.f("time_spacing");
    fmax_ = P_.f("max_frequency");
    if (nx_ <= 8 || nz_ <= 8) throw Error(FWI_ERR_PARAM, "x_samples and z_samples must exceed 8");
    if (!(dh_ > 0) || !(dt_ > 0) || !(fmax_ > 0) || nt_ < 2)
        throw Error(FWI_ERR_PARAM, "model_spacing, time_spacing, max_frequency must be positive, time_samples >= 2");
    idh2_ = 1.0f / (dh_ * dh_);
    seed_ = P_.u64_or("rbc_seed", 0);
    use_graphs_ = std::getenv("FWI2D_NO_GRAPHS") == nullptr;
    fwd_kernel_ = P_.str_or("fwd_kernel", "auto");
    if (const char* e = std::getenv("FWI2D_FWD_KERNEL")) fwd_kernel_ = e;
    bwd_kernel_ = P_.str_or("bwd_kernel", "auto");
    if (const char* e = std::getenv("FWI2D_BWD_KERNEL")) bwd_kernel_ = e;
    // test hooks of the bounded device waits (tests/test_gpu_failure.py)
    const uint64_t spin = P_.u64_or("test_wait_limit", 1u << 22);
    if (spin < 16 || spin > (1u << 22)) throw Error(FWI_ERR_PARAM, "test_wait_limit must lie in [16, 4194304]");
    spin_limit_ = (unsigned)spin;
    stall_fwd_ = P_.i_or("test_stall_fwd", -1);
    stall_bwd_ = P_.i_or("test_stall_bwd", -1);

    wavelet_ = make_wavelet(nt_, dt_, fmax_, &tlag_);
    geo_ = read_geometry(P_.str("SPS"), P_.str("RPS"));
    nsrc_ = geo_.nsrc();
    nrec_ = geo_.nrec();
    setup_windows();

    check(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");

    if (mode_ == FWI_MODE_MODELING || mode_ == FWI_MODE_INVERSION) {
        float abc_length = P_.f("abc_length");
        float abc_factor = P_.f("abc_factor");
        int nb = boundary_cells(abc_length, dh_);
        if (nb < 1) throw Error(FWI_ERR_PARAM, "abc_length gives no boundary cells");
        b1d_ = make_b1d(nb, abc_factor);
        setup_grid(&abc_, &abc_t_, nb);
        // ABC propagations read one shared padded model: a shot's grid is the
        // column range of it that starts at its window
        for (int s = 0; s < nsrc_; ++s) abc_t_.shots[s].vel_col = win_[s].c0;
        has_abc_ = true;
    }
    if (mode_ == FWI_MODE_MIGRATION || mode_ == FWI_MODE_INVERSION) {
        const std::string pre = mode_ == FWI_MODE_MIGRATION ? "mig_" : "inv_";
        rbc_ratio_ = P_.f(pre + "rbc_ratio");
        rbc_varVp_ = P_.f(pre + "rbc_varVp");
        float rbc_length = P_.f(pre + "rbc_length");
        if (!(rbc_ratio_ > 0)) throw Error(FWI_ERR_PARAM, pre + "rbc_ratio must be positive");
        setup_grid(&rbc_, &rbc_t_, boundary_cells(rbc_length, dh_));
        has_rbc_ = true;
    }
    range_n_ = nsrc_;
    if (mode_ == FWI_MODE_INVERSION) {
        zmask_ = P_.f("depth_mask");
        max_iteration_ = P_.i("max_iteration");
    }

    alloc_buffers();

    std::vector<float> vp((size_t)nx_ * nz_);
    read_floats(P_.str("model_file"), vp.data(), vp.size());
    set_model(vp.data());
}

void Engine::setup_windows() {
    std::vector<float> off;
    const std::string file = P_.str_or("aperture_file", "");
    const float one = P_.f_or("aperture_offset", 0.0f);
    if (!file.empty()) off = read_text_floats(file);
    else if (one > 0) off.assign(nsrc_, one);
    win_ = aperture_windows(geo_, nx_, dh_, off);
    windowed_ = !off.empty();
}

void Engine::setup_grid(Grid* g, Tables* t, int nb) {
    g->nb = nb;
    g->full_nxx = nx_ + 2 * nb;
    g->nzz = nz_ + 2 * nb;
    g->ldz = round_up(g->nzz, 32);
    g->nxx = 0;
    t->nxx.resize(nsrc_);
    for (int s = 0; s < nsrc_; ++s) {
        t->nxx[s] = win_[s].w + 2 * nb;
        g->nxx = std::max(g->nxx, t->nxx[s]);
    }
    // initialization, modeling.cu:252-277: indices on the padded whole model
    t->src_x.resize(nsrc_);
    t->src_z.resize(nsrc_);
    t->rec_x.resize(nrec_);
    t->rec_z.resize(nrec_);
    for (int s = 0; s < nsrc_; ++s) {
        t->src_x[s] = grid_index(geo_.xsrc[s], dh_, nb);
        t->src_z[s] = grid_index(geo_.zsrc[s], dh_, nb);
        const int lx = t->src_x[s] - win_[s].c0;
        if (lx < 0 || lx >= t->nxx[s] || t->src_z[s] < 0 || t->src_z[s] >= g->nzz)
            throw Error(FWI_ERR_PARAM, "source " + std::to_string(s + 1) + " lies outside the model");
    }
    for (int r = 0; r < nrec_; ++r) {
        t->rec_x[r] = grid_index(geo_.xrec[r], dh_, nb);
        t->rec_z[r] = grid_index(geo_.zrec[r], dh_, nb);
        if (!windowed_ && (t->rec_x[r] < 0 || t->rec_x[r] >= g->full_nxx || t->rec_z[r] < 0 || t->rec_z[r] >= g->nzz))
            throw Error(FWI_ERR_PARAM, "receiver " + std::to_string(r + 1) + " lies outside the model");
    }
    // receivers sorted by column (stable in receiver order)
    std::vector<int> order(nrec_);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return t->rec_x[a] < t->rec_x[b]; });
    t->shots.resize(nsrc_);
    std::vector<int> rec_pt, rec_colptr, rec_z, src_colptr, src_z(nsrc_);
    std::vector<long long> rec_soff, src_soff(nsrc_, 0);
    for (int s = 0; s < nsrc_; ++s) {
        const int nxx = t->nxx[s], c0 = win_[s].c0;
        ShotDesc& d = t->shots[s];
        d.nxx = nxx;
        d.rec_off = (int)rec_z.size();
        d.col_off = (int)src_colptr.size();
        d.seis_off = (long long)s * nrec_ * nt_;
        d.vel_col = 0;
        // source: one entry per shot, in the shot's own column table
        src_z[s] = t->src_z[s];
        const int sx = t->src_x[s] - c0;
        for (int j = 0; j <= nxx; ++j) src_colptr.push_back(s + (j > sx ? 1 : 0));
        // receivers of the shot's window (all of them without windows), by column
        std::vector<int> mine;
        for (int p = 0; p < nrec_; ++p) {
            const int r = order[p];
            const int m = t->rec_x[r] - nb;  // model column
            if (!windowed_ || (m >= c0 && m < c0 + win_[s].w && t->rec_z[r] >= 0 && t->rec_z[r] < g->nzz))
                mine.push_back(r);
        }
        d.nrec = (int)mine.size();
        int pos = 0;
        for (int j = 0; j <= nxx; ++j) {
            while (pos < d.nrec && t->rec_x[mine[pos]] - c0 < j) ++pos;
            rec_colptr.push_back(d.rec_off + pos);
        }
        for (int r : mine) {
            rec_z.push_back(t->rec_z[r]);
            rec_pt.push_back(t->rec_z[r] + (t->rec_x[r] - c0) * g->ldz);
            rec_soff.push_back(d.seis_off + (long long)r * nt_);
        }
    }
    auto up = [&](auto** dst, const auto& v, const char* what) {
        using T = std::remove_reference_t<decltype(v[0])>;
        *dst = dalloc<std::remove_const_t<T>>(std::max<size_t>(1, v.size()), what);
        if (!v.empty())
            check(cudaMemcpy(*dst, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice), what);
    };
    up(&t->d_rec_pt, rec_pt, "receiver points");
    up(&t->d_src_colptr, src_colptr, "source columns");
    up(&t->d_src_z, src_z, "source rows");
    up(&t->d_src_soff, src_soff, "source offsets");
    up(&t->d_rec_colptr, rec_colptr, "receiver columns");
    up(&t->d_rec_z, rec_z, "receiver rows");
    up(&t->d_rec_soff, rec_soff, "receiver offsets");
    t->h_src_colptr = std::move(src_colptr);
    t->h_rec_colptr = std::move(rec_colptr);
    t->h_rec_ent_z = rec_z;
    t->h_rec_ent_soff = rec_soff;
}

void Engine::free_tables(Tables* t) {
    cudaFree(t->d_rec_pt);
    cudaFree(t->d_src_colptr);
    cudaFree(t->d_src_z);
    cudaFree(t->d_src_soff);
    cudaFree(t->d_rec_colptr);
    cudaFree(t->d_rec_z);
    cudaFree(t->d_rec_soff);
}

void Engine::alloc_buffers() {
    const size_t npts = (size_t)nx_ * nz_;
    const size_t nseis = (size_t)nsrc_ * nrec_ * nt_;
    fstride_max_ = std::max(has_abc_ ? abc_.fstride() : 0LL, has_rbc_ ? rbc_.fstride() : 0LL);
    const int nfields = (mode_ == FWI_MODE_MODELING) ? 2 : 7;

    d_vp_ = dalloc<float>(npts, "velocity");
    d_tmp_ = dalloc<float>(npts, "scratch model");
    d_wavelet_ = dalloc<float>(nt_, "wavelet");
    check(cudaMemcpy(d_wavelet_, wavelet_.data(), nt_ * sizeof(float), cudaMemcpyHostToDevice), "upload wavelet");
    if (has_abc_) {
        d_b1d_ = dalloc<float>(b1d_.size(), "b1d");
        check(cudaMemcpy(d_b1d_, b1d_.data(), b1d_.size() * sizeof(float), cudaMemcpyHostToDevice), "upload b1d");
        d_vel_abc_ = dalloc<float>((size_t)abc_.ldz * abc_.full_nxx, "ABC velocity");
    }
    if (has_rbc_ && !windowed_) d_vel_rbc_base_ = dalloc<float>(rbc_.fstride(), "RBC base velocity");
    d_seis_ = dalloc<float>(nseis, "seismograms");
    if (mode_ != FWI_MODE_MODELING) d_data_ = dalloc<float>(nseis, "input data");
    if (mode_ == FWI_MODE_INVERSION) {
        d_res_ = dalloc<float>(nseis, "residuals");
        d_m_ = dalloc<float>(npts, "slowness^2");
        d_grad_ = dalloc<float>(npts, "gradient");
    }
    if (mode_ != FWI_MODE_MODELING) {
        d_img_ = dalloc<float>(npts, "image / raw gradient");
        d_illum_ = dalloc<float>(npts, "illumination");
        check(cudaMemset(d_img_, 0, npts * sizeof(float)), "memset image");
        check(cudaMemset(d_illum_, 0, npts * sizeof(float)), "memset illumination");
    }
    d_partial_ = dalloc<double>((size_t)residual_blocks((size_t)nrec_ * nt_ * std::max(1, nsrc_)) + 1, "partials");
    d_sum_ = dalloc<double>(1, "sum");
    d_flag_ = dalloc<int>(1, "flag");
    d_gmax_ = dalloc<unsigned int>(1, "gmax");

    // shots per batch: the key batch_shots, else what fits in half the free
    // memory.  Contexts that back-propagate cap a batch's field working set
    // at kBackwardBatchBytes and split the survey into equal batches: the
    // backward kernel streams seven fields, and on the B200 it ran at 0.80 /
    // 0.82 / 0.84 of the HBM bandwidth with 6 / 3 / 1.5 GB working sets (the
    // forward kernel loses about 2 % over the same range).
    size_t free_b = 0, total_b = 0;
    check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t per_shot = (size_t)nfields * (size_t)fstride_max_ * sizeof(float);
    size_t fit = per_shot ? (free_b / 2) / per_shot : (size_t)nsrc_;
    int want = P_.i_or("batch_shots", 0);
    batch_ = want > 0 ? want : (int)std::min<size_t>((size_t)nsrc_, std::max<size_t>(1, fit));
    if (want <= 0 && mode_ != FWI_MODE_MODELING && per_shot > 0) {
        constexpr size_t kBackwardBatchBytes = size_t(2) << 30;
        const int cap = (int)std::max<size_t>(1, kBackwardBatchBytes / per_shot);
        if (batch_ > cap) {
            const int nbatches = (nsrc_ + cap - 1) / cap;
            batch_ = std::min(batch_, (nsrc_ + nbatches - 1) / nbatches);
        }
    }
    batch_ = std::max(1, std::min(batch_, nsrc_));
    const size_t fsz = (size_t)batch_ * fstride_max_;
    for (int k = 0; k < kBufFields; ++k) fld_[k] = dalloc<float>(fsz, "wavefield");
    d_tile_base_ = dalloc<int>(batch_ + 1, "tile table");
    d_err_ = dalloc<int>(1, "error flag");
    d_sync_ = dalloc<unsigned>(1, "grid barrier");
    check(cudaMemset(d_err_, 0, sizeof(int)), "memset error flag");
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, dev), "SM count");
    if (mode_ != FWI_MODE_MODELING) {
        acc_[0] = dalloc<float>(fsz, "accumulator");
        acc_[1] = dalloc<float>(fsz, "illumination accumulator");
        d_vel_batch_ = dalloc<float>(fsz, "RBC velocity");
    }
    d_batch_ = dalloc<ShotDesc>(batch_, "batch descriptors");
    d_batch_nxx_ = dalloc<int>(nsrc_, "shot widths");
    d_batch_id_ = dalloc<int>(nsrc_, "shot ids");
    d_batch_c0_ = dalloc<int>(nsrc_, "window starts");
    d_batch_w_ = dalloc<int>(nsrc_, "window widths");
    d_bump_ptr_ = dalloc<int>(batch_ + 1, "bump offsets");
    std::vector<int> ids(nsrc_), c0(nsrc_), w(nsrc_), nxx(nsrc_);
    std::iota(ids.begin(), ids.end(), 0);
    for (int s = 0; s < nsrc_; ++s) {
        c0[s] = win_[s].c0;
        w[s] = win_[s].w;
        nxx[s] = has_rbc_ ? rbc_t_.nxx[s] : abc_t_.nxx[s];
    }
    {
        std::vector<float> geo;
        geo.insert(geo.end(), geo_.xsrc.begin(), geo_.xsrc.end());
        geo.insert(geo.end(), geo_.zsrc.begin(), geo_.zsrc.end());
        geo.insert(geo.end(), geo_.xrec.begin(), geo_.xrec.end());
        geo.insert(geo.end(), geo_.zrec.begin(), geo_.zrec.end());
        d_geo_ = dalloc<float>(geo.size(), "geometry");
        check(cudaMemcpy(d_geo_, geo.data(), geo.size() * sizeof(float), cudaMemcpyHostToDevice), "upload geometry");
        d_shot_bits_ = dalloc<unsigned>(nsrc_, "per-shot scratch");
        d_weights_ = dalloc<double>(1024, "filter weights");
    }
    const int full[2] = {0, nx_};
    d_full_win_ = dalloc<int>(2, "whole-model window");
    check(cudaMemcpy(d_full_win_, full, sizeof(full), cudaMemcpyHostToDevice), "upload whole-model window");
    if (windowed_ && mode_ == FWI_MODE_INVERSION) {
        // traces whose receiver lies outside the shot's window take no part in the misfit
        const Tables& t = has_abc_ ? abc_t_ : rbc_t_;
        std::vector<unsigned char> keep((size_t)nsrc_ * nrec_, 0);
        for (int s = 0; s < nsrc_; ++s)
            for (int r = 0; r < nrec_; ++r) {
                const int m = t.rec_x[r] - (has_abc_ ? abc_.nb : rbc_.nb);
                keep[(size_t)s * nrec_ + r] = (m >= win_[s].c0 && m < win_[s].c0 + win_[s].w) ? 1 : 0;
            }
        d_trace_keep_ = dalloc<unsigned char>(keep.size(), "trace mask");
        check(cudaMemcpy(d_trace_keep_, keep.data(), keep.size(), cudaMemcpyHostToDevice), "upload trace mask");
    }
    check(cudaMemcpy(d_batch_id_, ids.data(), nsrc_ * sizeof(int), cudaMemcpyHostToDevice), "upload ids");
    check(cudaMemcpy(d_batch_c0_, c0.data(), nsrc_ * sizeof(int), cudaMemcpyHostToDevice), "upload c0");
    check(cudaMemcpy(d_batch_w_, w.data(), nsrc_ * sizeof(int), cudaMemcpyHostToDevice), "upload w");
    check(cudaMemcpy(d_batch_nxx_, nxx.data(), nsrc_ * sizeof(int), cudaMemcpyHostToDevice), "upload nxx");
}

Engine::~Engine() {
    if (st_) cudaStreamSynchronize(st_);
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    if (has_abc_) free_tables(&abc_t_);
    if (has_rbc_) free_tables(&rbc_t_);
    void* ptrs[] = {d_vp_, d_m_, d_vel_abc_, d_vel_rbc_base_, d_wavelet_, d_b1d_, d_batch_, d_batch_nxx_,
                    d_batch_id_, d_batch_c0_, d_batch_w_, d_bump_ptr_, d_bumps_, fld_[0], fld_[1], fld_[2],
                    fld_[3], acc_[0], acc_[1], d_vel_batch_, d_seis_, d_data_, d_res_, d_partial_, d_sum_,
                    d_flag_, d_gmax_, d_img_, d_illum_, d_grad_, d_tmp_, d_tile_base_, d_err_, d_sync_,
                    d_slabs_, d_xbuf_, d_full_win_, d_trace_keep_, d_geo_, d_shot_bits_, d_weights_,
                    d_inj_ptr_, d_inj_pts_, d_inj_soff_, d_rec_ptr_, d_rec_pts_};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (auto& r : timed_) {
        event_pool_.push_back(r.begin);
        event_pool_.push_back(r.end);
    }
    for (cudaEvent_t e : event_pool_) cudaEventDestroy(e);
    if (st_) cudaStreamDestroy(st_);
}

// ---------------------------------------------------------------- kernel timing
void Engine::fwd_timing(bool enable) {
    double ms;
    long long l, u;
    fwd_timing_read(&ms, &l, &u);  // drain recorded regions
    timed_ms_ = btimed_ms_ = 0;
    timed_launches_ = timed_updates_ = btimed_launches_ = btimed_updates_ = 0;
    timing_ = enable;
}

cudaEvent_t Engine::timing_event() {
    if (!event_pool_.empty()) {
        cudaEvent_t e = event_pool_.back();
        event_pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    check(cudaEventCreate(&e), "create timing event");
    return e;
}

void Engine::timing_begin(TimedRegion* r) {
    if (!timing_) return;
    r->begin = timing_event();
    r->end = timing_event();
    check(cudaEventRecord(r->begin, st_), "record timing event");
}

void Engine::timing_end(TimedRegion* r, long long launches, long long updates) {
    if (!timing_ || !r->begin) return;
    check(cudaEventRecord(r->end, st_), "record timing event");
    r->launches = launches;
    r->updates = updates;
    timed_.push_back(*r);
}

void Engine::fwd_timing_read(double* ms, long long* launches, long long* updates) {
    for (auto& r : timed_) {
        check(cudaEventSynchronize(r.end), "timing event");
        float t = 0.f;
        check(cudaEventElapsedTime(&t, r.begin, r.end), "timing elapsed");
        if (r.launches >= 0) {
            timed_ms_ += t;
            timed_launches_ += r.launches;
            timed_updates_ += r.updates;
        } else {  // a backward region
            btimed_ms_ += t;
            btimed_launches_ -= r.launches;
            btimed_updates_ += r.updates;
        }
        event_pool_.push_back(r.begin);
        event_pool_.push_back(r.end);
    }
    timed_.clear();
    *ms = timed_ms_;
    *launches = timed_launches_;
    *updates = timed_updates_;
}

void Engine::bwd_timing_read(double* ms, long long* launches, long long* updates) {
    fwd_timing_read(ms, launches, updates);
    *ms = btimed_ms_;
    *launches = btimed_launches_;
    *updates = btimed_updates_;
}

fwi_dims Engine::dims() const {
    fwi_dims d;
    std::memset(&d, 0, sizeof(d));
    const Grid& g = has_abc_ ? abc_ : rbc_;
    d.nx = nx_;
    d.nz = nz_;
    d.nt = nt_;
    d.nsrc = nsrc_;
    d.nrec = nrec_;
    d.nb = g.nb;
    d.nxx = g.nxx;
    d.nzz = g.nzz;
    d.ldz = g.ldz;
    d.tlag = tlag_;
    d.abc_nb = has_abc_ ? abc_.nb : 0;
    d.rbc_nb = has_rbc_ ? rbc_.nb : 0;
    d.dh = dh_;
    d.dt = dt_;
    d.fmax = fmax_;
    d.vmin = vmin_;
    d.vmax = vmax_;
    return d;
}

// -------------------------------------------------------------------- model
void Engine::set_model(const float* vp) {
    const size_t n = (size_t)nx_ * nz_;
    float lo = 1e30f, hi = -1e30f;
    for (size_t k = 0; k < n; ++k) {
        if (!std::isfinite(vp[k]) || !(vp[k] > 0))
            throw Error(FWI_ERR_PARAM, "velocity model holds a non-positive or non-finite value at " + std::to_string(k));
        lo = std::min(lo, vp[k]);
        hi = std::max(hi, vp[k]);
    }
    const double vtop = (double)hi + (has_rbc_ ? std::max(0.0f, rbc_varVp_) : 0.0f);
    if (vtop * dt_ / dh_ > kCflLimit)
        throw Error(FWI_ERR_CFL, "unstable: (vmax" + std::string(has_rbc_ ? " + rbc_varVp" : "") + ")*dt/dh = " +
                                     std::to_string(vtop * dt_ / dh_) + " exceeds " + std::to_string(kCflLimit));
    vmin_ = lo;
    vmax_ = hi;
    check(cudaMemcpyAsync(d_vp_, vp, n * sizeof(float), cudaMemcpyHostToDevice, st_), "upload model");
    if (d_m_) {
        launch_slowness2(d_vp_, d_m_, n, st_);
        ++launches_;
    }
    vel_abc_valid_ = vel_rbc_valid_ = false;
    have_grad_ = false;
    sync("set_model");
}

void Engine::get_model(float* vp) {
    check(cudaMemcpyAsync(vp, d_vp_, (size_t)nx_ * nz_ * sizeof(float), cudaMemcpyDeviceToHost, st_), "get_model");
    sync("get_model");
}

void Engine::get_wavelet(float* w) const { std::memcpy(w, wavelet_.data(), wavelet_.size() * sizeof(float)); }

void Engine::get_indices(int shot, int* src_xz, int* rec_x, int* rec_z) const {
    if (shot < 0 || shot >= nsrc_) throw Error(FWI_ERR_ARG, "shot index out of range");
    const Tables& t = has_abc_ ? abc_t_ : rbc_t_;
    if (src_xz) {
        src_xz[0] = t.src_x[shot];
        src_xz[1] = t.src_z[shot];
    }
    if (rec_x) std::copy(t.rec_x.begin(), t.rec_x.end(), rec_x);
    if (rec_z) std::copy(t.rec_z.begin(), t.rec_z.end(), rec_z);
}

void Engine::expand_to(const Grid& g, const float* d_model, float* d_out) {
    launch_expand(d_model, nz_, nx_, d_out, 0, d_full_win_, d_full_win_ + 1, 1, g.nb, g.nzz, g.ldz, g.full_nxx, st_);
    ++launches_;
}

void Engine::get_window(int shot, int* c0, int* w) const {
    if (shot < 0 || shot >= nsrc_) throw Error(FWI_ERR_ARG, "shot index out of range");
    *c0 = win_[shot].c0;
    *w = win_[shot].w;
}

void Engine::rbc_base(int s0, int ns, const float** base, long long* stride) {
    if (!windowed_) {
        ensure_rbc_base();
        *base = d_vel_rbc_base_;
        *stride = 0;
        return;
    }
    // every shot's window, padded by edge replication, into the free
    // accumulator (the backward pass clears it before use)
    launch_expand(d_vp_, nz_, nx_, acc_[0], rbc_.fstride(), d_batch_c0_ + s0, d_batch_w_ + s0, ns, rbc_.nb, rbc_.nzz,
                  rbc_.ldz, rbc_.nxx, st_);
    ++launches_;
    *base = acc_[0];
    *stride = rbc_.fstride();
}

void Engine::ensure_rbc_base() {
    if (!vel_rbc_valid_) {
        expand_to(rbc_, d_vp_, d_vel_rbc_base_);
        vel_rbc_valid_ = true;
    }
}

// ------------------------------------------------------------------ batches
void Engine::upload_batch(const Tables& t, int s0, int ns) {
    batch_t_ = &t;
    batch_s0_ = s0;
    check(cudaMemcpyAsync(d_batch_, t.shots.data() + s0, ns * sizeof(ShotDesc), cudaMemcpyHostToDevice, st_),
          "upload batch");
    // the pageable source is staged before the call returns; the stream orders
    // the copy before the graph that reads it
}

void Engine::build_rbc(int s0, int ns) {
    const uint64_t seed_eff = seed_ + (uint64_t)rbc_epoch_ * kEpochStride;
    std::vector<std::vector<Bump>> per(ns);
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < ns; ++k)
        per[k] = make_bumps(rbc_t_.nxx[s0 + k], rbc_.nzz, rbc_.nb, dh_, rbc_ratio_, rbc_varVp_, seed_eff,
                            (uint32_t)(s0 + k));
    std::vector<int> ptr(ns + 1, 0);
    for (int k = 0; k < ns; ++k) ptr[k + 1] = ptr[k] + (int)per[k].size();
    std::vector<BumpDev> all((size_t)std::max(1, ptr[ns]));
    for (int k = 0; k < ns; ++k)
        for (size_t p = 0; p < per[k].size(); ++p) {
            const Bump& b = per[k][p];
            all[ptr[k] + p] = BumpDev{b.xc, b.zc, b.r, b.A, b.factor};
        }
    if (all.size() > bumps_cap_) {
        check(cudaStreamSynchronize(st_), "sync before bump realloc");
        cudaFree(d_bumps_);
        bumps_cap_ = all.size() * 2;
        d_bumps_ = dalloc<BumpDev>(bumps_cap_, "bumps");
    }
    check(cudaMemcpyAsync(d_bumps_, all.data(), all.size() * sizeof(BumpDev), cudaMemcpyHostToDevice, st_),
          "upload bumps");
    check(cudaMemcpyAsync(d_bump_ptr_, ptr.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice, st_),
          "upload bump offsets");
    RbcArgs a;
    rbc_base(s0, ns, &a.base, &a.base_stride);
    a.out = d_vel_batch_;
    a.out_stride = rbc_.fstride();
    a.nxx = d_batch_nxx_ + s0;
    a.shot_id = d_batch_id_ + s0;
    a.bumps = d_bumps_;
    a.bump_ptr = d_bump_ptr_;
    a.nzz = rbc_.nzz;
    a.ldz = rbc_.ldz;
    a.nb = rbc_.nb;
    a.max_nxx = rbc_.nxx;
    a.dh = dh_;
    a.varVp = rbc_varVp_;
    a.vmin = vmin_;
    a.vmax = vmax_;
    a.seed = seed_eff;
    launch_rbc(a, ns, st_);
    ++launches_;
    // bump vectors are pageable: synchronous staging makes them safe to drop
    check(cudaGetLastError(), "rbc launch");
}

// ------------------------------------------------------- TMA forward plans
namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
            throw Error(FWI_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}
}  // namespace

const CUtensorMap& Engine::tmap(const float* base, const Grid& g, int nshots, int boxz, int boxx, bool whole_model) {
    // whole_model: the shared padded model (nx + 2 nb columns, one "shot")
    const int width = whole_model ? g.full_nxx : g.nxx;
    const long long sstride = whole_model ? (long long)g.ldz * g.full_nxx : g.fstride();
    std::ostringstream k;
    k << (const void*)base << ':' << g.ldz << ':' << width << ':' << nshots << ':' << sstride << ':' << boxz << ':'
      << boxx;
    auto it = tmaps_.find(k.str());
    if (it != tmaps_.end()) return it->second;
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)g.ldz, (cuuint64_t)width, (cuuint64_t)nshots};
    cuuint64_t strides[2] = {(cuuint64_t)g.ldz * 4, (cuuint64_t)sstride * 4};
    cuuint32_t box[3] = {(cuuint32_t)boxz, (cuuint32_t)boxx, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
                             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(FWI_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return tmaps_.emplace(k.str(), m).first->second;
}

void Engine::upload_tile_base(const Grid& g, int ns, int tx) {
    const int ntz = (g.ldz + fwd_tma_rows() - 1) / fwd_tma_rows();
    std::vector<int> base(ns + 1, 0);
    for (int s = 0; s < ns; ++s) {
        const int nxx = h_shot_nxx(g, s);
        base[s + 1] = base[s] + ntz * ((nxx + tx - 1) / tx);
    }
    check(cudaMemcpyAsync(d_tile_base_, base.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice, st_),
          "upload tile table");
}

void Engine::launch_fwd_tma_step(const FwdPlan& p, bool two, const Grid& g, const Tables& t, int ns,
                                 const float* vel, long long vel_stride, bool abc, float* cur, float* old,
                                 float* out1, float* out2, int tt, bool record, float* d_seis) {
    // a one-level plan always runs its own variant; a two-level plan ends an
    // odd step count with its one-level tail variant
    const bool main_cfg = two || p.cfg.T == 1;
    const FwdTmaConfig& c = main_cfg ? p.cfg : p.tail;
    const int launch_grid = main_cfg ? p.grid : p.tail_grid;
    FwdTmaArgs a;
    a.shots = d_batch_;
    a.tile_base = d_tile_base_;
    a.ns = ns;
    a.ntz = (g.ldz + fwd_tma_rows() - 1) / fwd_tma_rows();
    a.ldz = g.ldz;
    a.nzz = g.nzz;
    a.nb = g.nb;
    a.fstride = g.fstride();
    a.vel_shared = vel_stride == 0 ? 1 : 0;
    a.dt2idh2 = dt_ * dt_ * idh2_;
    a.b1d = abc ? d_b1d_ : nullptr;
    a.inj = InjTable{t.d_src_colptr, t.d_src_z, t.d_src_soff, d_wavelet_, -1, idh2_};
    a.sample1 = (tt + 1 < nt_) ? tt + 1 : -1;
    a.sample2 = (two && tt + 2 < nt_) ? tt + 2 : -1;
    a.rec = InjTable{t.d_rec_colptr, t.d_rec_z, t.d_rec_soff, nullptr, -1, 0.0f};
    a.seis = record ? d_seis : nullptr;
    a.rec_sample0 = (record && tt > tlag_) ? tt - tlag_ : -1;
    a.rec_sample1 = (record && two && tt + 1 > tlag_) ? tt + 1 - tlag_ : -1;
    a.out1 = out1;
    a.out2 = out2;
    a.err = d_err_;
    a.spin = spin_limit_;
    a.stall = -1;
    const CUtensorMap& mc = tmap(cur, g, batch_, fwd_tma_box_cur_z(c), fwd_tma_box_cur_x(c));
    const CUtensorMap& mo = tmap(old, g, batch_, fwd_tma_box_pt_z(c), fwd_tma_box_pt_x(c));
    const CUtensorMap& mv =
        tmap(vel, g, vel_stride ? batch_ : 1, fwd_tma_box_pt_z(c), fwd_tma_box_pt_x(c), vel_stride == 0);
    check(launch_fwd_tma(c, mc, mo, mv, a, launch_grid, st_), "forward TMA launch");
}

double Engine::time_fwd_candidate(const FwdPlan& p, const Grid& g, const Tables& t, int ns, const float* vel,
                                  long long vel_stride, bool abc) {
    const long long fs = g.fstride();
    const dim3 grid = step_grid(g.ldz, g.nxx, ns);
    const int reps = 8;  // launches timed
    auto one = [&](int k) {
        if (p.kind == 0) {
            FwdArgs a;
            a.shots = d_batch_;
            a.vel = vel;
            a.vel_stride = vel_stride;
            a.cur = fld_[k % 2];
            a.nxt = fld_[(k + 1) % 2];
            a.fstride = fs;
            a.ldz = g.ldz;
            a.nzz = g.nzz;
            a.nb = g.nb;
            a.dt2idh2 = dt_ * dt_ * idh2_;
            a.b1d = abc ? d_b1d_ : nullptr;
            a.inj = InjTable{t.d_src_colptr, t.d_src_z, t.d_src_soff, d_wavelet_, -1, idh2_};
            a.rec_pt = t.d_rec_pt;
            a.rec_soff = t.d_rec_soff;
            a.seis = nullptr;
            a.rec_sample = -1;
            a.nt = nt_;
            launch_fwd_step(a, grid, st_);
        } else if (p.kind == 1) {
            upload_tile_base(g, ns, p.cfg.TX);
            launch_fwd_tma_step(p, p.cfg.T == 2, g, t, ns, vel, vel_stride, abc, fld_[k % 2], fld_[(k + 1) % 2],
                                fld_[2 + k % 2], fld_[3 - k % 2], 0, false, nullptr);
        }
    };
    const int loop_steps = 8 * reps;  // a multi-level launch is timed over more levels
    if (p.kind == 2) {
        upload_tile_base(g, ns, p.cfg.TX);
        launch_fwd_loop_levels(p, g, t, ns, vel, vel_stride, abc, false, nullptr, 0, 2);  // warm-up
    } else if (p.kind == 3) {
        launch_fwd_res_levels(p, g, t, vel, vel_stride, abc, nullptr, fld_[0], fld_[1], fld_[2], fld_[3], 0, 2);
    } else {
        one(0);  // first use: module load, tensor maps
    }
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    float ms = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {  // best of two timed runs
        check(cudaEventRecord(e0, st_), "event record");
        if (p.kind == 2) launch_fwd_loop_levels(p, g, t, ns, vel, vel_stride, abc, false, nullptr, 0, loop_steps);
        else if (p.kind == 3)
            launch_fwd_res_levels(p, g, t, vel, vel_stride, abc, nullptr, fld_[0], fld_[1], fld_[2], fld_[3], 0,
                                  loop_steps);
        else
            for (int k = 0; k < reps; ++k) one(k);
        check(cudaEventRecord(e1, st_), "event record");
        check(cudaEventSynchronize(e1), "event sync");
        float m = 0.f;
        cudaEventElapsedTime(&m, e0, e1);
        ms = std::min(ms, m);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int steps = p.kind >= 2 ? loop_steps : reps * (p.kind == 1 ? p.cfg.T : 1);
    return 1e3 * ms / steps;
}

void Engine::launch_fwd_loop_levels(const FwdPlan& p, const Grid& g, const Tables& t, int ns, const float* vel,
                                    long long vel_stride, bool abc, bool record, float* d_seis, int t_begin,
                                    int t_end, long long timed_updates) {
    const int TX = p.cfg.TX;
    FwdLoopMaps maps;
    for (int i = 0; i < 3; ++i) {
        maps.cur[i] = tmap(fld_[i], g, batch_, fwd_tma_rows() + 8, TX + 8);
        maps.pt[i] = tmap(fld_[i], g, batch_, fwd_tma_rows(), TX);
    }
    maps.cur[3] = maps.cur[2];
    maps.pt[3] = maps.pt[2];
    maps.vel = tmap(vel, g, vel_stride ? batch_ : 1, fwd_tma_rows(), TX, vel_stride == 0);
    FwdLoopArgs la;
    FwdTmaArgs& a = la.base;
    a.shots = d_batch_;
    a.tile_base = d_tile_base_;
    a.ns = ns;
    a.ntz = (g.ldz + fwd_tma_rows() - 1) / fwd_tma_rows();
    a.ldz = g.ldz;
    a.nzz = g.nzz;
    a.nb = g.nb;
    a.fstride = g.fstride();
    a.vel_shared = vel_stride == 0 ? 1 : 0;
    a.dt2idh2 = dt_ * dt_ * idh2_;
    a.b1d = abc ? d_b1d_ : nullptr;
    a.inj = InjTable{t.d_src_colptr, t.d_src_z, t.d_src_soff, d_wavelet_, -1, idh2_};
    a.sample1 = a.sample2 = -1;
    a.rec = InjTable{t.d_rec_colptr, t.d_rec_z, t.d_rec_soff, nullptr, -1, 0.0f};
    a.seis = record ? d_seis : nullptr;
    a.rec_sample0 = a.rec_sample1 = -1;
    a.out1 = a.out2 = nullptr;
    a.err = d_err_;
    a.spin = spin_limit_;
    a.stall = stall_fwd_;
    la.t_begin = t_begin;
    la.t_end = t_end;
    la.nt = nt_;
    la.tlag = tlag_;
    la.record = record ? 1 : 0;
    la.buf_cur = 0;
    la.buf_old = 1;
    la.buf_free = 2;
    for (int i = 0; i < 4; ++i) la.bufs[i] = fld_[i];
    la.sync = d_sync_;
    if (record) upload_record_points(g, t, ns, TX, p.grid);
    la.rec_cta_ptr = d_rec_ptr_;
    la.rec_pts = d_rec_pts_;
    check(cudaMemsetAsync(d_sync_, 0, sizeof(unsigned), st_), "memset grid barrier");
    TimedRegion r;
    if (timed_updates >= 0) timing_begin(&r);
    check(launch_fwd_loop(TX, p.cfg.S, p.minb, maps, la, p.grid, st_), "multi-level forward launch");
    if (timed_updates >= 0) timing_end(&r, 1, timed_updates);
    ++launches_;
}

bool Engine::plan_resident(const Grid& g, const Tables& t, int ns, FwdPlan* p) {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const size_t static_smem = fwd_res_static_smem();
    if ((size_t)optin <= static_smem) return false;
    const size_t max_dyn = (size_t)optin - static_smem;
    const int qg = g.ldz / 4;
    const size_t stage = fwd_res_stage_smem(g.ldz);  // halo staging, independent of the slab width
    const int wcap = max_dyn > stage ? (int)((max_dyn - stage) / (8 * (size_t)(g.ldz + 8))) - 8 : 0;
    std::vector<int> nxx(ns);
    for (int s = 0; s < ns; ++s) nxx[s] = h_shot_nxx(g, s);
    // slabs of at most W columns: per shot n slabs of equal width (a multiple
    // of 4, so that the edge runs are whole), the last taking the rest
    std::vector<ResSlab> slabs;
    int wmax = 0;
    auto build = [&](int W) {
        slabs.clear();
        wmax = 0;
        for (int s = 0; s < ns; ++s) {
            const int n = (nxx[s] + W - 1) / W;
            const int base = ((nxx[s] + n - 1) / n + 3) / 4 * 4;
            std::vector<int> w(n, base);
            w[n - 1] = nxx[s] - (n - 1) * base;
            if (n > 1 && w[n - 1] < 4) {
                w[n - 2] -= 4;
                w[n - 1] += 4;
            }
            const int first = (int)slabs.size();
            const ShotDesc& sd = t.shots[batch_s0_ + s];
            int x0 = 0;
            for (int k = 0; k < n; ++k) {
                if (w[k] < 4) return false;
                ResSlab sl{};
                sl.s = s;
                sl.x0 = x0;
                sl.w = w[k];
                sl.left = k > 0 ? first + k - 1 : -1;
                sl.right = k + 1 < n ? first + k + 1 : -1;
                const int a = sd.col_off + x0, b = sd.col_off + x0 + w[k];
                if (t.h_rec_colptr[b] - t.h_rec_colptr[a] > fwd_res_max_rec()) return false;
                if (t.h_src_colptr[b] - t.h_src_colptr[a] > fwd_res_max_src()) return false;
                slabs.push_back(sl);
                x0 += w[k];
                wmax = std::max(wmax, w[k]);
            }
        }
        return true;
    };
    // the narrowest slab width whose slabs fit one per SM
    bool found = false;
    for (int W = 4; W <= wcap && !found; W += 4) {
        long long total = 0;
        for (int s = 0; s < ns; ++s) total += (nxx[s] + W - 1) / W;
        found = total <= sm_count_ && build(W);
    }
    if (!found) return false;
    const long long items = (long long)((wmax + 3) / 4) * qg;
    const int ipt = (int)((items + fwd_res_threads() - 1) / fwd_res_threads());
    const size_t smem = fwd_res_smem((wmax + 3) / 4 * 4, g.ldz);
    if (!fwd_res_fits(wmax, g.ldz) || smem > max_dyn) return false;
    int ctas = 0;
    if (fwd_res_configure(g.ldz, smem, &ctas) != cudaSuccess || ctas < 1) {
        cudaGetLastError();
        return false;
    }
    if ((long long)slabs.size() > (long long)sm_count_ * ctas) return false;
    p->ipt = ipt;
    p->wmax = (wmax + 3) / 4 * 4;  // buffer columns: whole 4-column runs
    p->smem = smem;
    p->grid = (int)slabs.size();
    p->slabs = std::move(slabs);
    return true;
}

void Engine::launch_fwd_res_levels(const FwdPlan& p, const Grid& g, const Tables& t, const float* vel,
                                   long long vel_stride, bool abc, float* d_seis, const float* in_cur,
                                   const float* in_old, float* out_cur, float* out_old, int t_begin, int t_end,
                                   long long timed_updates) {
    const size_t nsl = p.slabs.size();
    // 16-byte words: 2 parities x 2 sides x 2 ldz per slab, and one slab's
    // worth more (the failure drill's stalled slab publishes there)
    const size_t xb = (size_t)8 * (nsl + 1) * g.ldz;
    if (nsl > slabs_cap_ || xb > xbuf_cap_) {
        check(cudaStreamSynchronize(st_), "sync before resident-kernel tables");
        cudaFree(d_slabs_);
        cudaFree(d_xbuf_);
        d_slabs_ = nullptr;
        d_xbuf_ = nullptr;
        slabs_cap_ = std::max(slabs_cap_, nsl);
        xbuf_cap_ = std::max(xbuf_cap_, xb);
        d_slabs_ = dalloc<ResSlab>(slabs_cap_, "slab table");
        d_xbuf_ = dalloc<ulonglong2>(xbuf_cap_, "halo exchange buffer");
    }
    check(cudaMemcpyAsync(d_slabs_, p.slabs.data(), nsl * sizeof(ResSlab), cudaMemcpyHostToDevice, st_),
          "upload slab table");
    FwdResArgs a;
    a.shots = d_batch_;
    a.slabs = d_slabs_;
    a.nslab = (int)nsl;
    a.wmax = p.wmax;
    a.ldz = g.ldz;
    a.nzz = g.nzz;
    a.nb = g.nb;
    a.fstride = g.fstride();
    a.vel = vel;
    a.vel_stride = vel_stride;
    a.dt2idh2 = dt_ * dt_ * idh2_;
    a.b1d = abc ? d_b1d_ : nullptr;
    a.inj = InjTable{t.d_src_colptr, t.d_src_z, t.d_src_soff, d_wavelet_, -1, idh2_};
    a.rec = InjTable{t.d_rec_colptr, t.d_rec_z, t.d_rec_soff, nullptr, -1, 0.0f};
    a.seis = d_seis;
    a.t_begin = t_begin;
    a.t_end = t_end;
    a.nt = nt_;
    a.tlag = tlag_;
    a.in_cur = in_cur;
    a.in_old = in_old;
    a.out_cur = out_cur;
    a.out_old = out_old;
    a.xbuf = d_xbuf_;
    a.err = d_err_;
    a.spin = spin_limit_;
    a.stall = stall_fwd_;
    check(cudaMemsetAsync(d_xbuf_, 0, xb * sizeof(ulonglong2), st_), "memset halo exchange buffer");
    TimedRegion r;
    if (timed_updates >= 0) timing_begin(&r);
    check(launch_fwd_res(a, p.smem, st_), "resident forward launch");
    if (timed_updates >= 0) timing_end(&r, 1, timed_updates);
    ++launches_;
}

Engine::FwdPlan Engine::fwd_plan(const Grid& g, const Tables& t, int ns, bool abc, const float* vel,
                                 long long vel_stride) {
    const long long key = ((long long)(&g == &abc_ ? 0 : 1) * 2 + (abc ? 1 : 0)) * 4 * 1000000LL +
                          (vel_stride ? 1000000LL : 0) + ns;
    auto it = plans_.find(key);
    if (it != plans_.end()) return it->second;
    auto make = [&](int T, int TX, int S) {
        FwdPlan p;
        p.kind = 1;
        p.cfg = FwdTmaConfig{T, TX, S};
        p.tail = FwdTmaConfig{1, TX, TX == 32 ? 2 : 3};
        int ctas = 0, ctas_t = 0;
        if (fwd_tma_configure(&ctas, p.cfg) != cudaSuccess || ctas < 1) {
            cudaGetLastError();
            p.kind = -1;
            return p;
        }
        if (fwd_tma_configure(&ctas_t, p.tail) != cudaSuccess || ctas_t < 1) {
            cudaGetLastError();
            p.kind = -1;
            return p;
        }
        p.grid = sm_count_ * ctas;
        p.tail_grid = sm_count_ * ctas_t;
        return p;
    };
    auto make_loop = [&](int TX, int S, int B) {
        FwdPlan p;
        p.kind = 2;
        p.cfg = FwdTmaConfig{1, TX, S};
        p.minb = B;
        int ctas = 0;
        if (fwd_loop_configure(&ctas, TX, S, B) != cudaSuccess || ctas < 1) {
            cudaGetLastError();
            p.kind = -1;
            return p;
        }
        p.grid = sm_count_ * ctas;
        return p;
    };
    auto make_res = [&]() {
        FwdPlan p;
        p.kind = 3;
        if (!plan_resident(g, t, ns, &p)) p.kind = -1;
        return p;
    };
    std::vector<FwdPlan> cands;
    if (fwd_kernel_ == "resident") {
        cands.push_back(make_res());
        if (cands.back().kind < 0)
            throw Error(FWI_ERR_PARAM, "fwd_kernel 'resident': the batch's fields do not fit the SMs' shared memory");
    } else if (fwd_kernel_ == "simple") {
        cands.push_back(FwdPlan{});
    } else if (fwd_kernel_.rfind("tma:", 0) == 0) {
        int T = 0, TX = 0, S = 0;
        if (std::sscanf(fwd_kernel_.c_str() + 4, "%d,%d,%d", &T, &TX, &S) != 3 || !fwd_tma_supported({T, TX, S}))
            throw Error(FWI_ERR_PARAM, "fwd_kernel '" + fwd_kernel_ + "' is not a compiled TMA variant");
        cands.push_back(make(T, TX, S));
    } else if (fwd_kernel_.rfind("loop:", 0) == 0) {
        int TX = 0, S = 0, B = 2;
        const int got = std::sscanf(fwd_kernel_.c_str() + 5, "%d,%d,%d", &TX, &S, &B);
        if (got < 2 || !fwd_loop_supported(TX, S, B))
            throw Error(FWI_ERR_PARAM, "fwd_kernel '" + fwd_kernel_ + "' is not a compiled multi-level variant");
        cands.push_back(make_loop(TX, S, B));
    } else if (fwd_kernel_ == "auto" || fwd_kernel_ == "tma") {
        if (fwd_kernel_ == "auto") cands.push_back(FwdPlan{});
        const int variants[][3] = {{1, 32, 2}, {1, 32, 3}, {1, 16, 3}, {1, 16, 4}, {2, 32, 2}, {2, 16, 2}, {2, 16, 3}};
        for (const auto& v : variants) cands.push_back(make(v[0], v[1], v[2]));
        const int loops[][3] = {{32, 2, 2}, {16, 3, 2}, {16, 2, 2}, {16, 2, 3}};
        for (const auto& v : loops) cands.push_back(make_loop(v[0], v[1], v[2]));
        cands.push_back(make_res());
    } else {
        throw Error(FWI_ERR_PARAM, "fwd_kernel must be auto, simple, tma, tma:T,TX,S, loop:TX,S[,B] or resident");
    }
    FwdPlan best;
    double best_us = 1e30;
    std::ostringstream log;
    for (auto& c : cands) {
        if (c.kind < 0) continue;
        if (cands.size() == 1) {
            best = c;
            break;
        }
        c.us_per_step = time_fwd_candidate(c, g, t, ns, vel, vel_stride, abc);
        if (c.kind == 0) log << " simple=" << c.us_per_step;
        else if (c.kind == 2) log << " loop" << c.cfg.TX << "," << c.cfg.S << "," << c.minb << "=" << c.us_per_step;
        else if (c.kind == 3) log << " resident=" << c.us_per_step;
        else log << " tma" << c.cfg.T << "," << c.cfg.TX << "," << c.cfg.S << "=" << c.us_per_step;
        if (c.us_per_step < best_us) {
            best_us = c.us_per_step;
            best = c;
        }
    }
    sync("forward autotune");
    best.tuning = log.str();
    plans_[key] = best;
    return best;
}

void Engine::run_forward(const Grid& g, const Tables& t, int ns, const float* vel, long long vel_stride, bool abc,
                         bool record, float* d_seis) {
    const long long fs = g.fstride();
    const FwdPlan plan = fwd_plan(g, t, ns, abc, vel, vel_stride);
    {
        std::ostringstream d;
        if (plan.kind == 0) d << "simple";
        else if (plan.kind == 2)
            d << "loop TX=" << plan.cfg.TX << " S=" << plan.cfg.S << " B=" << plan.minb << " grid=" << plan.grid;
        else if (plan.kind == 3)
            d << "resident W=" << plan.wmax << " IPT=" << plan.ipt << " grid=" << plan.grid;
        else d << "tma T=" << plan.cfg.T << " TX=" << plan.cfg.TX << " S=" << plan.cfg.S << " grid=" << plan.grid;
        if (!plan.tuning.empty()) d << " | us/step:" << plan.tuning;
        last_fwd_plan = d.str();
    }
    float* B[4] = {fld_[0], fld_[1], fld_[2], fld_[3]};
    check(cudaMemsetAsync(B[0], 0, (size_t)ns * fs * sizeof(float), st_), "memset field");
    check(cudaMemsetAsync(B[1], 0, (size_t)ns * fs * sizeof(float), st_), "memset field");
    InjTable inj{t.d_src_colptr, t.d_src_z, t.d_src_soff, d_wavelet_, 0, idh2_};
    launch_inject_points(B[0], fs, d_batch_, ns, inj, g.ldz, st_);
    ++launches_;
    const int N = nt_ + tlag_;
    if (plan.kind == 3) {
        // every level in one cooperative launch, the fields resident in shared memory
        launch_fwd_res_levels(plan, g, t, vel, vel_stride, abc, record ? d_seis : nullptr, B[0], B[1], B[2], B[3], 0,
                              N, (long long)N * batch_points(g, ns));
        fwd_cur_ = B[2];
        fwd_old_ = B[3];
        check(cudaGetLastError(), "forward propagation");
        return;
    }
    if (plan.kind == 2) {
        // every level in one cooperative launch: buffers rotate cur -> old, free -> cur
        upload_tile_base(g, ns, plan.cfg.TX);
        launch_fwd_loop_levels(plan, g, t, ns, vel, vel_stride, abc, record, d_seis, 0, N,
                               (long long)N * batch_points(g, ns));
        int c = 0, o = 1, f = 2;
        for (int tt = 0; tt < N; ++tt) {
            const int po = o;
            o = c;
            c = f;
            f = po;
        }
        fwd_cur_ = B[c];
        fwd_old_ = B[o];
        check(cudaGetLastError(), "forward propagation");
        return;
    }
    const dim3 grid = step_grid(g.ldz, g.nxx, ns);
    const float dt2idh2 = dt_ * dt_ * idh2_;
    int launches_in_loop = 0;
    // buffer roles after the loop (indices into B)
    int cur = 0, old = 1;
    if (plan.kind == 1) {
        upload_tile_base(g, ns, plan.cfg.TX);
        int f0 = 2, f1 = 3, tt = 0;
        cur = 0;
        old = 1;
        while (tt < N) {
            const bool two = plan.cfg.T == 2 && tt + 1 < N;
            const int pc = cur, po = old;
            if (two) {
                old = f0;
                cur = f1;
                f0 = pc;
                f1 = po;
                tt += 2;
            } else {
                old = pc;
                cur = f0;
                f0 = po;
                tt += 1;
            }
            ++launches_in_loop;
        }
    } else {
        cur = N % 2;
        old = (N + 1) % 2;
        launches_in_loop = N;
    }
    auto body = [&]() {
        if (plan.kind == 1) {
            int c = 0, o = 1, f0 = 2, f1 = 3, tt = 0;
            while (tt < N) {
                const bool two = plan.cfg.T == 2 && tt + 1 < N;
                launch_fwd_tma_step(plan, two, g, t, ns, vel, vel_stride, abc, B[c], B[o], B[f0], two ? B[f1] : nullptr,
                                    tt, record, d_seis);
                const int pc = c, po = o;
                if (two) {
                    o = f0;
                    c = f1;
                    f0 = pc;
                    f1 = po;
                    tt += 2;
                } else {
                    o = pc;
                    c = f0;
                    f0 = po;
                    tt += 1;
                }
            }
            return;
        }
        for (int tt = 0; tt < N; ++tt) {
            FwdArgs a;
            a.shots = d_batch_;
            a.vel = vel;
            a.vel_stride = vel_stride;
            a.cur = (tt % 2 == 0) ? B[0] : B[1];
            a.nxt = (tt % 2 == 0) ? B[1] : B[0];
            a.fstride = fs;
            a.ldz = g.ldz;
            a.nzz = g.nzz;
            a.nb = g.nb;
            a.dt2idh2 = dt2idh2;
            a.b1d = abc ? d_b1d_ : nullptr;
            a.inj = inj;
            a.inj.sample = (tt + 1 < nt_) ? tt + 1 : -1;
            a.rec_pt = t.d_rec_pt;
            a.rec_soff = t.d_rec_soff;
            a.seis = d_seis;
            a.rec_sample = (record && tt > tlag_) ? tt - tlag_ : -1;
            a.nt = nt_;
            launch_fwd_step(a, grid, st_);
        }
    };
    fwd_cur_ = B[cur];
    fwd_old_ = B[old];
    const long long key = ((((long long)(record ? kFwdRecord : kFwdNoRecord) * 2 + (abc ? 0 : 1)) * 4 +
                            (&g == &abc_ ? 0 : 1)) * 8 + (vel_stride ? 1 : 0)) * 1000000LL + ns;
    if (use_graphs_) {
        auto it = graphs_.find(key);
        if (it == graphs_.end()) {
            cudaGraph_t graph;
            check(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal), "begin capture");
            body();
            check(cudaStreamEndCapture(st_, &graph), "end capture");
            cudaGraphExec_t exec;
            check(cudaGraphInstantiate(&exec, graph, 0), "instantiate graph");
            cudaGraphDestroy(graph);
            it = graphs_.emplace(key, exec).first;
        }
        TimedRegion r;
        timing_begin(&r);
        check(cudaGraphLaunch(it->second, st_), "graph launch");
        timing_end(&r, launches_in_loop, (long long)N * batch_points(g, ns));
    } else {
        TimedRegion r;
        timing_begin(&r);
        body();
        timing_end(&r, launches_in_loop, (long long)N * batch_points(g, ns));
    }
    launches_ += launches_in_loop;
    check(cudaGetLastError(), "forward propagation");
}

Engine::BwdPlan Engine::bwd_plan(const Grid& g, const Tables& t, int ns, const float* vel, long long vel_stride,
                                 bool gradient, const float* d_series, float* scratch0, float* scratch1) {
    const long long key = (((long long)(&g == &abc_ ? 0 : 1) * 2 + (gradient ? 1 : 0)) * 2 + (vel_stride ? 1 : 0)) *
                              1000000LL + ns;
    auto it = bwd_plans_.find(key);
    if (it != bwd_plans_.end()) return it->second;
    auto make_loop = [&](int TX, int S) {
        BwdPlan p;
        p.kind = 2;
        p.TX = TX;
        p.S = S;
        int ctas = 0;
        if (bwd_loop_configure(&ctas, TX, S) != cudaSuccess || ctas < 1) {
            cudaGetLastError();
            p.kind = -1;
            return p;
        }
        p.grid = sm_count_ * ctas;
        return p;
    };
    std::vector<BwdPlan> cands;
    if (bwd_kernel_ == "simple") {
        cands.push_back(BwdPlan{});
    } else if (bwd_kernel_.rfind("loop:", 0) == 0) {
        int TX = 0, S = 0;
        if (std::sscanf(bwd_kernel_.c_str() + 5, "%d,%d", &TX, &S) != 2 || !bwd_loop_supported(TX, S))
            throw Error(FWI_ERR_PARAM, "bwd_kernel '" + bwd_kernel_ + "' is not a compiled multi-level variant");
        cands.push_back(make_loop(TX, S));
    } else if (bwd_kernel_ == "auto") {
        cands.push_back(BwdPlan{});
        const int loops[][2] = {{16, 3}, {16, 2}, {8, 4}, {8, 3}};
        for (const auto& v : loops) cands.push_back(make_loop(v[0], v[1]));
    } else {
        throw Error(FWI_ERR_PARAM, "bwd_kernel must be auto, simple or loop:TX,S");
    }
    // Candidates run on scratch buffers only (the forward's final fields stay
    // untouched): both fields alias scratch0/scratch1, the accumulators are
    // cleared by the caller afterwards.
    BwdPlan best;
    double best_us = 1e30;
    std::ostringstream log;
    const int levels = 24;
    float* ps[2] = {scratch0, scratch1};
    float* pr[2] = {scratch1, scratch0};
    const dim3 grid = step_grid(g.ldz, g.nxx, ns);
    for (auto& c : cands) {
        if (c.kind < 0) continue;
        if (cands.size() == 1) {
            best = c;
            break;
        }
        auto run = [&](int nlev) {
            if (c.kind == 2) {
                upload_tile_base(g, ns, c.TX);
                launch_bwd_loop_levels(c, g, t, ns, vel, vel_stride, gradient, d_series, ps, pr, 0, nlev);
                return;
            }
            for (int b = 0; b < nlev; ++b) {
                BwdArgs a;
                a.shots = d_batch_;
                a.vel = vel;
                a.vel_stride = vel_stride;
                a.ps_st = ps[(b + 1) & 1];
                a.ps_io = ps[b & 1];
                a.pr_st = pr[b & 1];
                a.pr_io = pr[(b + 1) & 1];
                a.fstride = g.fstride();
                a.acc_a = acc_[0];
                a.acc_b = acc_[1];
                a.acc_stride = g.fstride();
                a.ldz = g.ldz;
                a.nzz = g.nzz;
                a.dt2idh2 = dt_ * dt_ * idh2_;
                a.dt = dt_;
                a.idh2 = idh2_;
                a.inj = InjTable{t.d_rec_colptr, t.d_rec_z, t.d_rec_soff, d_series, nt_ - 2 - b, idh2_};
                if (a.inj.sample < 0) a.inj.sample = -1;
                launch_bwd_step(a, gradient, grid, st_);
            }
        };
        run(2);  // first use
        cudaEvent_t e0, e1;
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
        float ms = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            check(cudaEventRecord(e0, st_), "event record");
            run(levels);
            check(cudaEventRecord(e1, st_), "event record");
            check(cudaEventSynchronize(e1), "event sync");
            float m = 0.f;
            cudaEventElapsedTime(&m, e0, e1);
            ms = std::min(ms, m);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c.us_per_step = 1e3 * ms / levels;
        if (c.kind == 0) log << " simple=" << c.us_per_step;
        else log << " loop" << c.TX << "," << c.S << "=" << c.us_per_step;
        if (c.us_per_step < best_us) {
            best_us = c.us_per_step;
            best = c;
        }
    }
    sync("backward autotune");
    best.tuning = log.str();
    bwd_plans_[key] = best;
    return best;
}

// Receiver points of the batch's shots per CTA of a multi-level backward
// launch of `grid` CTAs over tx-column tiles: tiles are numbered as in
// upload_tile_base (down the columns of a shot, shots in order) and CTA b owns
// tiles b, b + grid, ...; entries at the same point stay together, in entry
// order, so one thread adds them as the column-table walk did.
void Engine::upload_injection_points(const Grid& g, const Tables& t, int ns, int tx, int grid) {
    const int R = fwd_tma_rows();
    const int ntz = (g.ldz + R - 1) / R;
    const long long fs = g.fstride();
    struct Rec {
        int cta;
        long long g;
        int k;
    };
    std::vector<Rec> recs;
    int tile0 = 0;
    for (int s = 0; s < ns; ++s) {
        const ShotDesc& sd = t.shots[batch_s0_ + s];
        const int nxx = h_shot_nxx(g, s);
        for (int j = 0; j < nxx; ++j) {
            const int kb = t.h_rec_colptr[sd.col_off + j], ke = t.h_rec_colptr[sd.col_off + j + 1];
            for (int k = kb; k < ke; ++k) {
                const int z = t.h_rec_ent_z[k];
                const int tile = tile0 + (j / tx) * ntz + z / R;
                recs.push_back(Rec{tile % grid, (long long)s * fs + (long long)j * g.ldz + z, k});
            }
        }
        tile0 += ntz * ((nxx + tx - 1) / tx);
    }
    std::sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) {
        return a.cta != b.cta ? a.cta < b.cta : (a.g != b.g ? a.g < b.g : a.k < b.k);
    });
    h_inj_ptr_.assign((size_t)grid + 1, 0);
    h_inj_pts_.clear();
    h_inj_soff_.clear();
    for (size_t i = 0; i < recs.size();) {
        InjPoint pt;
        pt.g = recs[i].g;
        pt.e0 = (int)h_inj_soff_.size();
        size_t e = i;
        for (; e < recs.size() && recs[e].cta == recs[i].cta && recs[e].g == recs[i].g; ++e)
            h_inj_soff_.push_back(t.h_rec_ent_soff[recs[e].k]);
        pt.e1 = (int)h_inj_soff_.size();
        h_inj_pts_.push_back(pt);
        ++h_inj_ptr_[recs[i].cta + 1];
        i = e;
    }
    for (int b = 0; b < grid; ++b) h_inj_ptr_[b + 1] += h_inj_ptr_[b];
    auto grow = [&](auto** buf, size_t* cap, size_t need, const char* what) {
        using T = std::remove_pointer_t<std::remove_reference_t<decltype(*buf)>>;
        need = std::max<size_t>(need, 1);
        if (need > *cap) {
            check(cudaStreamSynchronize(st_), "sync before injection-table realloc");
            cudaFree(*buf);
            *buf = nullptr;
            *cap = 0;
            *buf = dalloc<T>(need * 2, what);
            *cap = need * 2;
        }
    };
    grow(&d_inj_ptr_, &inj_ptr_cap_, h_inj_ptr_.size(), "injection CTA table");
    grow(&d_inj_pts_, &inj_pts_cap_, h_inj_pts_.size(), "injection points");
    grow(&d_inj_soff_, &inj_soff_cap_, h_inj_soff_.size(), "injection trace offsets");
    check(cudaMemcpyAsync(d_inj_ptr_, h_inj_ptr_.data(), h_inj_ptr_.size() * sizeof(int), cudaMemcpyHostToDevice,
                          st_),
          "upload injection CTA table");
    if (!h_inj_pts_.empty()) {
        check(cudaMemcpyAsync(d_inj_pts_, h_inj_pts_.data(), h_inj_pts_.size() * sizeof(InjPoint),
                              cudaMemcpyHostToDevice, st_),
              "upload injection points");
        check(cudaMemcpyAsync(d_inj_soff_, h_inj_soff_.data(), h_inj_soff_.size() * sizeof(long long),
                              cudaMemcpyHostToDevice, st_),
              "upload injection trace offsets");
    }
}

// Receiver entries of the batch's shots per CTA of a multi-level forward
// launch (tiles numbered as in upload_tile_base, CTA b owns tiles b, b + grid,
// ...), in entry order within a CTA.
void Engine::upload_record_points(const Grid& g, const Tables& t, int ns, int tx, int grid) {
    const int R = fwd_tma_rows();
    const int ntz = (g.ldz + R - 1) / R;
    const long long fs = g.fstride();
    std::vector<std::pair<int, RecPoint>> recs;
    int tile0 = 0;
    for (int s = 0; s < ns; ++s) {
        const ShotDesc& sd = t.shots[batch_s0_ + s];
        const int nxx = h_shot_nxx(g, s);
        for (int j = 0; j < nxx; ++j) {
            const int kb = t.h_rec_colptr[sd.col_off + j], ke = t.h_rec_colptr[sd.col_off + j + 1];
            for (int k = kb; k < ke; ++k) {
                const int z = t.h_rec_ent_z[k];
                const int tile = tile0 + (j / tx) * ntz + z / R;
                recs.emplace_back(tile % grid,
                                  RecPoint{(long long)s * fs + (long long)j * g.ldz + z, t.h_rec_ent_soff[k], z, j, nxx, 0});
            }
        }
        tile0 += ntz * ((nxx + tx - 1) / tx);
    }
    std::stable_sort(recs.begin(), recs.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    h_rec_ptr_.assign((size_t)grid + 1, 0);
    h_rec_pts_.clear();
    for (const auto& r : recs) {
        ++h_rec_ptr_[r.first + 1];
        h_rec_pts_.push_back(r.second);
    }
    for (int b = 0; b < grid; ++b) h_rec_ptr_[b + 1] += h_rec_ptr_[b];
    auto grow = [&](auto** buf, size_t* cap, size_t need, const char* what) {
        using T = std::remove_pointer_t<std::remove_reference_t<decltype(*buf)>>;
        need = std::max<size_t>(need, 1);
        if (need > *cap) {
            check(cudaStreamSynchronize(st_), "sync before record-table realloc");
            cudaFree(*buf);
            *buf = nullptr;
            *cap = 0;
            *buf = dalloc<T>(need * 2, what);
            *cap = need * 2;
        }
    };
    grow(&d_rec_ptr_, &rec_ptr_cap_, h_rec_ptr_.size(), "record CTA table");
    grow(&d_rec_pts_, &rec_pts_cap_, h_rec_pts_.size(), "record points");
    check(cudaMemcpyAsync(d_rec_ptr_, h_rec_ptr_.data(), h_rec_ptr_.size() * sizeof(int), cudaMemcpyHostToDevice,
                          st_),
          "upload record CTA table");
    if (!h_rec_pts_.empty())
        check(cudaMemcpyAsync(d_rec_pts_, h_rec_pts_.data(), h_rec_pts_.size() * sizeof(RecPoint),
                              cudaMemcpyHostToDevice, st_),
              "upload record points");
}

void Engine::launch_bwd_loop_levels(const BwdPlan& p, const Grid& g, const Tables& t, int ns, const float* vel,
                                    long long vel_stride, bool gradient, const float* d_series, float* const ps[2],
                                    float* const pr[2], int b_begin, int b_end, long long timed_updates) {
    const int R = fwd_tma_rows();
    BwdLoopMaps maps;
    for (int q = 0; q < 2; ++q) {
        maps.ps_st[q] = tmap(ps[q ^ 1], g, batch_, R + 8, p.TX + 8);
        maps.pr_st[q] = tmap(pr[q], g, batch_, R + 8, p.TX + 8);
        maps.ps_pt[q] = tmap(ps[q], g, batch_, R, p.TX);
        maps.pr_pt[q] = tmap(pr[q ^ 1], g, batch_, R, p.TX);
    }
    maps.acc_a = tmap(acc_[0], g, batch_, R, p.TX);
    maps.acc_b = tmap(acc_[1], g, batch_, R, p.TX);
    maps.vel = tmap(vel, g, vel_stride ? batch_ : 1, R, p.TX, vel_stride == 0);
    BwdLoopArgs a;
    a.shots = d_batch_;
    a.tile_base = d_tile_base_;
    a.ns = ns;
    a.ntz = (g.ldz + R - 1) / R;
    a.ldz = g.ldz;
    a.nzz = g.nzz;
    a.fstride = g.fstride();
    a.vel_shared = vel_stride == 0 ? 1 : 0;
    a.dt2idh2 = dt_ * dt_ * idh2_;
    a.dt = dt_;
    a.idh2 = idh2_;
    a.inj = InjTable{t.d_rec_colptr, t.d_rec_z, t.d_rec_soff, d_series, -1, idh2_};
    a.nt = nt_;
    a.b_begin = b_begin;
    a.b_end = b_end;
    a.ps[0] = ps[0];
    a.ps[1] = ps[1];
    a.pr[0] = pr[0];
    a.pr[1] = pr[1];
    a.acc_a = acc_[0];
    a.acc_b = acc_[1];
    upload_injection_points(g, t, ns, p.TX, p.grid);
    a.inj_cta_ptr = d_inj_ptr_;
    a.inj_pts = d_inj_pts_;
    a.inj_soff = d_inj_soff_;
    a.err = d_err_;
    a.sync = d_sync_;
    a.spin = spin_limit_;
    a.stall = stall_bwd_;
    check(cudaMemsetAsync(d_sync_, 0, sizeof(unsigned), st_), "memset grid barrier");
    TimedRegion r;
    if (timed_updates >= 0) timing_begin(&r);
    check(launch_bwd_loop(p.TX, p.S, gradient, maps, a, p.grid, st_), "multi-level backward launch");
    if (timed_updates >= 0) timing_end(&r, -1, timed_updates);
    ++launches_;
}

void Engine::run_backward(const Grid& g, const Tables& t, int ns, const float* vel, long long vel_stride,
                          bool gradient, const float* d_series) {
    const long long fs = g.fstride();
    const int N = nt_ + tlag_;
    float* X = fwd_cur_;  // Q^N      (Ps of migration.cu:76)
    float* Y = fwd_old_;  // Q^{N-1}  (Psold)
    float* free_buf[2];
    int nf = 0;
    for (float* b : fld_)
        if (b != X && b != Y && nf < 2) free_buf[nf++] = b;
    float* R0 = free_buf[0];
    float* R1 = free_buf[1];
    const BwdPlan plan = bwd_plan(g, t, ns, vel, vel_stride, gradient, d_series, R0, R1);
    {
        std::ostringstream d;
        if (plan.kind == 2) d << "loop TX=" << plan.TX << " S=" << plan.S << " grid=" << plan.grid;
        else d << "simple";
        if (!plan.tuning.empty()) d << " | us/step:" << plan.tuning;
        last_bwd_plan = d.str();
    }
    const size_t bytes = (size_t)ns * fs * sizeof(float);
    check(cudaMemsetAsync(R0, 0, bytes, st_), "memset Pr");
    check(cudaMemsetAsync(R1, 0, bytes, st_), "memset Prold");
    check(cudaMemsetAsync(acc_[0], 0, bytes, st_), "memset accumulator");
    check(cudaMemsetAsync(acc_[1], 0, bytes, st_), "memset accumulator");
    InjTable inj{t.d_rec_colptr, t.d_rec_z, t.d_rec_soff, d_series, nt_ - 1, idh2_};
    launch_inject_points(R0, fs, d_batch_, ns, inj, g.ldz, st_);
    ++launches_;
    if (plan.kind == 2) {
        upload_tile_base(g, ns, plan.TX);
        float* ps[2] = {X, Y};
        float* pr[2] = {R0, R1};
        launch_bwd_loop_levels(plan, g, t, ns, vel, vel_stride, gradient, d_series, ps, pr, 0, N,
                               (long long)N * batch_points(g, ns));
        check(cudaGetLastError(), "backward propagation");
        return;
    }
    const dim3 grid = step_grid(g.ldz, g.nxx, ns);
    const float dt2idh2 = dt_ * dt_ * idh2_;
    auto body = [&]() {
        for (int b = 0; b < N; ++b) {
            BwdArgs a;
            a.shots = d_batch_;
            a.vel = vel;
            a.vel_stride = vel_stride;
            a.ps_st = (b % 2 == 0) ? Y : X;
            a.ps_io = (b % 2 == 0) ? X : Y;
            a.pr_st = (b % 2 == 0) ? R0 : R1;
            a.pr_io = (b % 2 == 0) ? R1 : R0;
            a.fstride = fs;
            a.acc_a = acc_[0];
            a.acc_b = acc_[1];
            a.acc_stride = fs;
            a.ldz = g.ldz;
            a.nzz = g.nzz;
            a.dt2idh2 = dt2idh2;
            a.dt = dt_;
            a.idh2 = idh2_;
            a.inj = inj;
            a.inj.sample = (b + 1 < nt_) ? nt_ - 1 - (b + 1) : -1;
            launch_bwd_step(a, gradient, grid, st_);
        }
    };
    int xi = 0, yi = 0;
    for (int k = 0; k < kBufFields; ++k) {
        if (fld_[k] == X) xi = k;
        if (fld_[k] == Y) yi = k;
    }
    const long long key =
        (((long long)(gradient ? kBwdGradient : kBwdImage) * 8 + 4 + (&g == &abc_ ? 0 : 1)) * 16 + xi * 4 + yi) *
            1000000LL + ns;
    TimedRegion r;
    if (use_graphs_) {
        auto it = graphs_.find(key);
        if (it == graphs_.end()) {
            cudaGraph_t graph;
            check(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal), "begin capture");
            body();
            check(cudaStreamEndCapture(st_, &graph), "end capture");
            cudaGraphExec_t exec;
            check(cudaGraphInstantiate(&exec, graph, 0), "instantiate graph");
            cudaGraphDestroy(graph);
            it = graphs_.emplace(key, exec).first;
        }
        timing_begin(&r);
        check(cudaGraphLaunch(it->second, st_), "graph launch");
    } else {
        timing_begin(&r);
        body();
    }
    timing_end(&r, -(long long)N, (long long)N * batch_points(g, ns));
    launches_ += N;
    check(cudaGetLastError(), "backward propagation");
}

void Engine::check_finite(const float* d, size_t n, const char* what) {
    check(cudaMemsetAsync(d_flag_, 0, sizeof(int), st_), "memset flag");
    launch_check_finite(d, n, d_flag_, st_);
    ++launches_;
    int flag = 0;
    check(cudaMemcpyAsync(&flag, d_flag_, sizeof(int), cudaMemcpyDeviceToHost, st_), "read flag");
    sync(what);
    if (flag) throw Error(FWI_ERR_NAN, std::string(what) + ": non-finite values (unstable propagation?)");
}

// ---------------------------------------------------------------- modeling
void Engine::model_shots(int s0, int ns, float* out, bool out_on_device) {
    if (!has_abc_) throw Error(FWI_ERR_STATE, "modeling needs a context created for modeling or inversion");
    if (s0 < 0 || ns < 0 || s0 + ns > nsrc_) throw Error(FWI_ERR_ARG, "shot range out of bounds");
    if (ns == 0) return;
    if (!vel_abc_valid_) {
        expand_to(abc_, d_vp_, d_vel_abc_);
        vel_abc_valid_ = true;
    }
    const size_t per = (size_t)nrec_ * nt_;
    check(cudaMemsetAsync(d_seis_ + (size_t)s0 * per, 0, (size_t)ns * per * sizeof(float), st_), "memset seis");
    for (int b0 = s0; b0 < s0 + ns; b0 += batch_) {
        const int nb = std::min(batch_, s0 + ns - b0);
        upload_batch(abc_t_, b0, nb);
        run_forward(abc_, abc_t_, nb, d_vel_abc_, 0, true, true, d_seis_);
    }
    check_finite(d_seis_ + (size_t)s0 * per, (size_t)ns * per, "modeling");
    if (out) {
        check(cudaMemcpyAsync(out, d_seis_ + (size_t)s0 * per, (size_t)ns * per * sizeof(float),
                              out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st_),
              "copy seismograms");
    }
    sync("model_shots");
}

// --------------------------------------------------------------- migration
void Engine::rtm_reset() {
    if (!has_rbc_) throw Error(FWI_ERR_STATE, "migration needs a context created for migration or inversion");
    const size_t n = (size_t)nx_ * nz_;
    check(cudaMemsetAsync(d_img_, 0, n * sizeof(float), st_), "memset image");
    check(cudaMemsetAsync(d_illum_, 0, n * sizeof(float), st_), "memset illumination");
    sync("rtm_reset");
}

void Engine::rtm_shots(int s0, int ns, const float* data, bool data_on_device) {
    if (!has_rbc_) throw Error(FWI_ERR_STATE, "migration needs a context created for migration or inversion");
    if (s0 < 0 || ns < 0 || s0 + ns > nsrc_) throw Error(FWI_ERR_ARG, "shot range out of bounds");
    if (ns == 0) return;
    const size_t per = (size_t)nrec_ * nt_;
    if (data)
        check(cudaMemcpyAsync(d_data_ + (size_t)s0 * per, data, (size_t)ns * per * sizeof(float),
                              data_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st_),
              "upload migration data");
    for (int b0 = s0; b0 < s0 + ns; b0 += batch_) {
        const int nb = std::min(batch_, s0 + ns - b0);
        upload_batch(rbc_t_, b0, nb);
        build_rbc(b0, nb);
        run_forward(rbc_, rbc_t_, nb, d_vel_batch_, rbc_.fstride(), false, false, d_seis_);
        run_backward(rbc_, rbc_t_, nb, d_vel_batch_, rbc_.fstride(), false, d_data_);
        launch_crop_sum(acc_[0], rbc_.fstride(), nb, rbc_.nb, rbc_.ldz, nz_, nx_, d_batch_c0_ + b0, d_batch_w_ + b0,
                        d_img_, true, st_);
        launch_crop_sum(acc_[1], rbc_.fstride(), nb, rbc_.nb, rbc_.ldz, nz_, nx_, d_batch_c0_ + b0, d_batch_w_ + b0,
                        d_illum_, true, st_);
        launches_ += 2;
    }
    check_finite(d_img_, (size_t)nx_ * nz_, "migration");
}

void Engine::rtm_image(float* image) {
    if (!has_rbc_) throw Error(FWI_ERR_STATE, "no migration state");
    launch_rtm_post(d_img_, d_illum_, nz_, nx_, idh2_, d_tmp_, st_);
    ++launches_;
    check(cudaMemcpyAsync(image, d_tmp_, (size_t)nx_ * nz_ * sizeof(float), cudaMemcpyDeviceToHost, st_),
          "copy image");
    sync("rtm_image");
}

void Engine::rtm_raw(float* img, float* illum) {
    if (!has_rbc_) throw Error(FWI_ERR_STATE, "no migration state");
    const size_t n = (size_t)nx_ * nz_ * sizeof(float);
    if (img) check(cudaMemcpyAsync(img, d_img_, n, cudaMemcpyDeviceToHost, st_), "copy image");
    if (illum) check(cudaMemcpyAsync(illum, d_illum_, n, cudaMemcpyDeviceToHost, st_), "copy illumination");
    sync("rtm_raw");
}

// ---------------------------------------------------------- data preparation
void Engine::mute_direct(float* data, bool on_device, float velocity, float delay, float gstd) {
    if (!data) throw Error(FWI_ERR_ARG, "NULL data");
    if (!(velocity > 0) || !(dt_ > 0) || !(gstd > 0)) throw Error(FWI_ERR_ARG, "velocity and gstd must be positive");
    const size_t n = (size_t)nsrc_ * nrec_ * nt_;
    float* d = data;
    if (!on_device) {
        d = d_seis_;
        check(cudaMemcpyAsync(d, data, n * sizeof(float), cudaMemcpyHostToDevice, st_), "upload data");
    }
    launch_mute_direct(d, nsrc_, nrec_, nt_, d_geo_, d_geo_ + nsrc_, d_geo_ + 2 * nsrc_, d_geo_ + 2 * nsrc_ + nrec_,
                       velocity, delay, dt_, gstd, d_shot_bits_, st_);
    launches_ += 2;
    if (!on_device) check(cudaMemcpyAsync(data, d, n * sizeof(float), cudaMemcpyDeviceToHost, st_), "copy data");
    sync("mute_direct");
}

void Engine::smooth_model(const float* vp, float sigma, float depth_mask, float* out) {
    if (!vp || !out) throw Error(FWI_ERR_ARG, "NULL model");
    if (!(sigma > 0)) throw Error(FWI_ERR_ARG, "sigma must be positive");
    // scipy.ndimage gaussian_filter1d kernel: radius int(4 sigma + 0.5),
    // exp(-0.5 x^2 / sigma^2) normalised by its numpy (pairwise) sum
    const double sd = sigma;
    const int radius = (int)(4.0 * sd + 0.5);
    if (radius >= 1024) throw Error(FWI_ERR_ARG, "sigma too large");
    std::vector<double> phi(2 * radius + 1);
    for (int k = -radius; k <= radius; ++k) phi[k + radius] = std::exp(-0.5 / (sd * sd) * (double)k * (double)k);
    double sum;
    const size_t m = phi.size();
    if (m < 8) {
        sum = 0.0;
        for (double x : phi) sum += x;
    } else {  // numpy's pairwise_sum for n <= 128: 8 partial sums, then the tail
        double r[8];
        for (int j = 0; j < 8; ++j) r[j] = phi[j];
        size_t i = 8;
        for (; i < m - m % 8; i += 8)
            for (int j = 0; j < 8; ++j) r[j] += phi[i + j];
        sum = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < m; ++i) sum += phi[i];
    }
    std::vector<double> half(radius + 1);
    for (int k = 0; k <= radius; ++k) half[k] = phi[radius + k] / sum;
    const size_t n = (size_t)nx_ * nz_;
    const int keep = std::max(0, (int)((double)depth_mask / (double)dh_));
    // scratch for the input, the z-pass and the result (freed on every exit)
    std::unique_ptr<float, decltype(&cudaFree)> buf(dalloc<float>(3 * n, "smoothing scratch"), &cudaFree);
    float* d_in = buf.get();
    check(cudaMemcpyAsync(d_weights_, half.data(), half.size() * sizeof(double), cudaMemcpyHostToDevice, st_),
          "upload weights");
    check(cudaMemcpyAsync(d_in, vp, n * sizeof(float), cudaMemcpyHostToDevice, st_), "upload model");
    launch_smooth_slowness(d_in, nz_, nx_, d_weights_, radius, keep, d_in + n, d_in + 2 * n, st_);
    launches_ += 3;
    check(cudaMemcpyAsync(out, d_in + 2 * n, n * sizeof(float), cudaMemcpyDeviceToHost, st_), "copy model");
    sync("smooth_model");
}

void Engine::random_boundary(int shot, float* out) {
    if (!has_rbc_) throw Error(FWI_ERR_STATE, "no random-boundary grid in this context");
    if (shot < 0 || shot >= nsrc_) throw Error(FWI_ERR_ARG, "shot index out of range");
    upload_batch(rbc_t_, shot, 1);
    build_rbc(shot, 1);
    std::vector<float> pitched((size_t)rbc_.fstride());
    check(cudaMemcpyAsync(pitched.data(), d_vel_batch_, pitched.size() * sizeof(float), cudaMemcpyDeviceToHost, st_),
          "copy random boundary");
    sync("random_boundary");
    for (int j = 0; j < rbc_t_.nxx[shot]; ++j)
        std::memcpy(out + (size_t)j * rbc_.nzz, pitched.data() + (size_t)j * rbc_.ldz, rbc_.nzz * sizeof(float));
}

// ---------------------------------------------------------------- inversion
void Engine::set_observed(const float* obs, bool on_device) {
    if (mode_ != FWI_MODE_INVERSION) throw Error(FWI_ERR_STATE, "observed data needs an inversion context");
    const size_t n = (size_t)nsrc_ * nrec_ * nt_;
    check(cudaMemcpyAsync(d_data_, obs, n * sizeof(float),
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st_),
          "upload observed data");
    if (d_trace_keep_) {
        launch_mask_traces(d_data_, d_trace_keep_, (size_t)nsrc_ * nrec_, nt_, st_);
        ++launches_;
    }
    sync("set_observed");
    have_obs_ = true;
}

double Engine::residual_of(int s0, int ns, const float* d_obs, const float* d_cal, float* d_res) {
    const size_t per = (size_t)nrec_ * nt_;
    const size_t off = (size_t)s0 * per, n = (size_t)ns * per;
    launch_residual(d_obs + off, d_cal + off, d_res + off, n, d_partial_, d_sum_, st_);
    launches_ += 2;
    double h = 0.0;
    check(cudaMemcpyAsync(&h, d_sum_, sizeof(double), cudaMemcpyDeviceToHost, st_), "read misfit");
    sync("residual");
    return h;
}

void Engine::set_shot_range(int s0, int ns) {
    if (s0 < 0 || ns < 0 || s0 + ns > nsrc_) throw Error(FWI_ERR_ARG, "shot range out of bounds");
    range_s0_ = s0;
    range_n_ = ns;
}

void Engine::accumulators(float** a, float** b) const {
    if (!d_img_) throw Error(FWI_ERR_STATE, "no image / gradient accumulators in a modeling context");
    *a = d_img_;
    *b = d_illum_;
}

double Engine::accumulate_gradient(bool with_gradient) {
    if (mode_ != FWI_MODE_INVERSION) throw Error(FWI_ERR_STATE, "gradient needs an inversion context");
    if (!have_obs_) throw Error(FWI_ERR_STATE, "observed data not set");
    const size_t npts = (size_t)nx_ * nz_;
    if (!vel_abc_valid_) {
        expand_to(abc_, d_vp_, d_vel_abc_);
        vel_abc_valid_ = true;
    }
    if (with_gradient) {
        check(cudaMemsetAsync(d_img_, 0, npts * sizeof(float), st_), "memset gradient");
        check(cudaMemsetAsync(d_illum_, 0, npts * sizeof(float), st_), "memset illumination");
    }
    const size_t per = (size_t)nrec_ * nt_;
    double sum = 0.0;
    const int s_end = range_s0_ + range_n_;
    for (int b0 = range_s0_; b0 < s_end; b0 += batch_) {
        const int nb = std::min(batch_, s_end - b0);
        check(cudaMemsetAsync(d_seis_ + (size_t)b0 * per, 0, (size_t)nb * per * sizeof(float), st_), "memset seis");
        upload_batch(abc_t_, b0, nb);
        run_forward(abc_, abc_t_, nb, d_vel_abc_, 0, true, true, d_seis_);
        sum += residual_of(b0, nb, d_data_, d_seis_, d_res_);
        if (with_gradient) {
            upload_batch(rbc_t_, b0, nb);
            build_rbc(b0, nb);
            run_forward(rbc_, rbc_t_, nb, d_vel_batch_, rbc_.fstride(), false, false, d_seis_);
            run_backward(rbc_, rbc_t_, nb, d_vel_batch_, rbc_.fstride(), true, d_res_);
            launch_crop_sum(acc_[0], rbc_.fstride(), nb, rbc_.nb, rbc_.ldz, nz_, nx_, d_batch_c0_ + b0,
                            d_batch_w_ + b0, d_img_, true, st_);
            launch_crop_sum(acc_[1], rbc_.fstride(), nb, rbc_.nb, rbc_.ldz, nz_, nx_, d_batch_c0_ + b0,
                            d_batch_w_ + b0, d_illum_, true, st_);
            launches_ += 2;
        }
    }
    if (with_gradient) ++rbc_epoch_;
    sync("accumulate_gradient");
    if (!std::isfinite(sum))
        throw Error(FWI_ERR_NAN, "accumulate_gradient: non-finite misfit (the model's propagation is unstable: a "
                                 "velocity above the CFL limit or a non-positive slowness^2 after an update?)");
    return sum;
}

void Engine::finish_gradient() {
    if (mode_ != FWI_MODE_INVERSION) throw Error(FWI_ERR_STATE, "gradient needs an inversion context");
    const size_t npts = (size_t)nx_ * nz_;
    launch_grad_post(d_img_, d_illum_, nz_, nx_, idh2_, (int)(zmask_ / dh_), d_grad_, d_gmax_, st_);
    launch_scale_by_inverse(d_grad_, npts, d_gmax_, st_);
    launches_ += 2;
    have_grad_ = true;
    sync("finish_gradient");
}

double Engine::compute_gradient(bool with_gradient) {
    const double sum = accumulate_gradient(with_gradient);
    if (with_gradient) finish_gradient();
    return sum;
}

void Engine::set_direction(const float* dir, bool on_device) {
    if (mode_ != FWI_MODE_INVERSION) throw Error(FWI_ERR_STATE, "a search direction needs an inversion context");
    if (!dir) throw Error(FWI_ERR_ARG, "NULL direction");
    const size_t n = (size_t)nx_ * nz_;
    check(cudaMemcpyAsync(d_grad_, dir, n * sizeof(float),
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st_),
          "set direction");
    launch_absmax(d_grad_, n, d_gmax_, st_);
    launch_scale_by_inverse(d_grad_, n, d_gmax_, st_);
    launches_ += 2;
    have_grad_ = true;
    sync("set_direction");
}

void Engine::get_gradient(float* g) {
    if (!have_grad_) throw Error(FWI_ERR_STATE, "no gradient computed");
    check(cudaMemcpyAsync(g, d_grad_, (size_t)nx_ * nz_ * sizeof(float), cudaMemcpyDeviceToHost, st_), "copy gradient");
    sync("get_gradient");
}

void Engine::get_gradient_raw(float* g, float* illum) {
    if (mode_ != FWI_MODE_INVERSION) throw Error(FWI_ERR_STATE, "no gradient in this context");
    const size_t n = (size_t)nx_ * nz_ * sizeof(float);
    if (g) check(cudaMemcpyAsync(g, d_img_, n, cudaMemcpyDeviceToHost, st_), "copy raw gradient");
    if (illum) check(cudaMemcpyAsync(illum, d_illum_, n, cudaMemcpyDeviceToHost, st_), "copy illumination");
    sync("get_gradient_raw");
}

double Engine::linesearch_trial(float alpha) {
    if (!have_grad_) throw Error(FWI_ERR_STATE, "no gradient computed");
    const size_t npts = (size_t)nx_ * nz_;
    launch_trial_velocity(d_m_, d_grad_, alpha, d_tmp_, npts, st_);
    ++launches_;
    expand_to(abc_, d_tmp_, d_vel_abc_);
    vel_abc_valid_ = false;  // holds the trial model now
    const size_t per = (size_t)nrec_ * nt_;
    double sum = 0.0;
    const int s_end = range_s0_ + range_n_;
    for (int b0 = range_s0_; b0 < s_end; b0 += batch_) {
        const int nb = std::min(batch_, s_end - b0);
        check(cudaMemsetAsync(d_seis_ + (size_t)b0 * per, 0, (size_t)nb * per * sizeof(float), st_), "memset seis");
        upload_batch(abc_t_, b0, nb);
        run_forward(abc_, abc_t_, nb, d_vel_abc_, 0, true, true, d_seis_);
        sum += residual_of(b0, nb, d_data_, d_seis_, d_res_);
    }
    return sum;
}

void Engine::trial_steps(float* a1, float* a2) const {
    // inversion.cu:288-293, in float as there
    const float dm = (1.0f / (vmin_ * vmin_)) - (1.0f / (vmax_ * vmax_));
    *a1 = 0.02f * dm;
    *a2 = 0.05f * dm;
}

float Engine::parabola_step(float f0, float f1, float f2) const {
    // inversion.cu:300-307, in float as there
    float a1, a2;
    trial_steps(&a1, &a2);
    const float a0 = 0.00f * ((1.0f / (vmin_ * vmin_)) - (1.0f / (vmax_ * vmax_)));
    float num = (a1 * a1 - a2 * a2) * f0 + (a2 * a2 - a0 * a0) * f1 + (a0 * a0 - a1 * a1) * f2;
    float den = (a1 - a2) * f0 + (a2 - a0) * f1 + (a0 - a1) * f2;
    return 0.5f * (num / den);
}

float Engine::optimization(float f0) {
    // inversion.cu:286-308, in float as there
    float dm = (1.0f / (vmin_ * vmin_)) - (1.0f / (vmax_ * vmax_));
    float a0 = 0.00f * dm;
    float a1 = 0.02f * dm;
    float a2 = 0.05f * dm;
    float f1 = sqrtf((float)linesearch_trial(a1));
    float f2 = sqrtf((float)linesearch_trial(a2));
    float num = (a1 * a1 - a2 * a2) * f0 + (a2 * a2 - a0 * a0) * f1 + (a0 * a0 - a1 * a1) * f2;
    float den = (a1 - a2) * f0 + (a2 - a0) * f1 + (a0 - a1) * f2;
    return 0.5f * (num / den);
}

void Engine::update_model(float step, float* vp_out, float vmin, float vmax) {
    if (!have_grad_) throw Error(FWI_ERR_STATE, "no gradient computed");
    if (vmin != 0.0f && !(vmin > 0.0f && vmax > vmin)) throw Error(FWI_ERR_ARG, "bounds need 0 < vmin < vmax");
    const size_t npts = (size_t)nx_ * nz_;
    const float mlo = vmin > 0.0f ? 1.0f / (vmax * vmax) : 0.0f;
    const float mhi = vmin > 0.0f ? 1.0f / (vmin * vmin) : 0.0f;
    launch_update_model(d_m_, d_grad_, step, d_vp_, npts, st_, mlo, mhi);
    ++launches_;
    vel_abc_valid_ = vel_rbc_valid_ = false;
    if (vp_out) check(cudaMemcpyAsync(vp_out, d_vp_, npts * sizeof(float), cudaMemcpyDeviceToHost, st_), "copy model");
    sync("update_model");
}

}  // namespace fwi
