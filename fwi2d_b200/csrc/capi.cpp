// capi.cpp — extern "C" surface of fwi2d.h over fwi::Engine.  Every entry
// point catches exceptions and turns them into status codes; the message is
// kept per context (or per thread for failures of fwi_ctx_create).
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>

#include "../../include/fwi2d.h"
#include "detmath.h"
#include "engine.hpp"

struct fwi_ctx {
    fwi::Engine* eng = nullptr;
    std::string err;
};

namespace {
thread_local std::string g_create_error;

template <typename F>
int guarded(fwi_ctx* ctx, F&& f) {
    if (!ctx || !ctx->eng) return FWI_ERR_ARG;
    try {
        f(*ctx->eng);
        ctx->err.clear();
        return FWI_OK;
    } catch (const fwi::Error& e) {
        ctx->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        ctx->err = "host allocation failed";
        return FWI_ERR_NOMEM;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return FWI_ERR_PARAM;
    }
}

int arg_error(fwi_ctx* ctx, const char* msg) {
    if (ctx) ctx->err = msg;
    return FWI_ERR_ARG;
}
}  // namespace

extern "C" {

int fwi_ctx_create(const char* params_path, int mode, fwi_ctx** out) {
    if (!out || !params_path) {
        g_create_error = "NULL argument";
        return FWI_ERR_ARG;
    }
    *out = nullptr;
    try {
        auto* c = new fwi_ctx();
        try {
            c->eng = new fwi::Engine(params_path, mode);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
        g_create_error.clear();
        return FWI_OK;
    } catch (const fwi::Error& e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return FWI_ERR_PARAM;
    }
}

void fwi_ctx_destroy(fwi_ctx* ctx) {
    if (!ctx) return;
    delete ctx->eng;
    delete ctx;
}

const char* fwi_last_error(const fwi_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int fwi_get_dims(const fwi_ctx* ctx, fwi_dims* out) {
    if (!ctx || !ctx->eng || !out) return FWI_ERR_ARG;
    *out = ctx->eng->dims();
    return FWI_OK;
}

int fwi_get_stream(const fwi_ctx* ctx, void** stream) {
    if (!ctx || !ctx->eng || !stream) return FWI_ERR_ARG;
    *stream = (void*)ctx->eng->stream();
    return FWI_OK;
}

int fwi_get_param(const fwi_ctx* ctx, const char* key, char* buf, size_t len) {
    if (!ctx || !ctx->eng || !key || !buf) return FWI_ERR_ARG;
    try {
        std::string v = ctx->eng->params().str(key);
        if (v.size() + 1 > len) return FWI_ERR_ARG;
        std::memcpy(buf, v.c_str(), v.size() + 1);
        return FWI_OK;
    } catch (const fwi::Error& e) {
        return e.code;
    }
}

int fwi_set_seed(fwi_ctx* ctx, uint64_t seed) {
    return guarded(ctx, [&](fwi::Engine& e) { e.set_seed(seed); });
}

int fwi_set_model(fwi_ctx* ctx, const float* vp) {
    if (!vp) return arg_error(ctx, "NULL model");
    return guarded(ctx, [&](fwi::Engine& e) { e.set_model(vp); });
}

int fwi_get_model(fwi_ctx* ctx, float* vp) {
    if (!vp) return arg_error(ctx, "NULL model");
    return guarded(ctx, [&](fwi::Engine& e) { e.get_model(vp); });
}

int fwi_get_wavelet(fwi_ctx* ctx, float* w) {
    if (!w) return arg_error(ctx, "NULL wavelet");
    return guarded(ctx, [&](fwi::Engine& e) { e.get_wavelet(w); });
}

int fwi_get_indices(fwi_ctx* ctx, int shot, int* src_xz, int* rec_x, int* rec_z) {
    return guarded(ctx, [&](fwi::Engine& e) { e.get_indices(shot, src_xz, rec_x, rec_z); });
}

int fwi_get_window(fwi_ctx* ctx, int shot, int* c0, int* w) {
    if (!c0 || !w) return arg_error(ctx, "NULL window output");
    return guarded(ctx, [&](fwi::Engine& e) { e.get_window(shot, c0, w); });
}

int fwi_model_shot(fwi_ctx* ctx, int shot, float* seis) {
    if (!seis) return arg_error(ctx, "NULL seismogram");
    return guarded(ctx, [&](fwi::Engine& e) { e.model_shots(shot, 1, seis, false); });
}

int fwi_model_survey(fwi_ctx* ctx, float* seis_all) {
    return guarded(ctx, [&](fwi::Engine& e) {
        e.model_shots(e.range_s0(), e.range_n(), seis_all ? seis_all + e.survey_offset(e.range_s0()) : nullptr, false);
    });
}

int fwi_model_survey_dev(fwi_ctx* ctx, float* d_seis_all) {
    return guarded(ctx, [&](fwi::Engine& e) {
        e.model_shots(e.range_s0(), e.range_n(), d_seis_all ? d_seis_all + e.survey_offset(e.range_s0()) : nullptr,
                      true);
    });
}

int fwi_rtm_reset(fwi_ctx* ctx) {
    return guarded(ctx, [&](fwi::Engine& e) { e.rtm_reset(); });
}

int fwi_rtm_shot(fwi_ctx* ctx, int shot, const float* data) {
    if (!data) return arg_error(ctx, "NULL data");
    return guarded(ctx, [&](fwi::Engine& e) { e.rtm_shots(shot, 1, data, false); });
}

int fwi_rtm_survey(fwi_ctx* ctx, const float* data_all) {
    if (!data_all) return arg_error(ctx, "NULL data");
    return guarded(ctx, [&](fwi::Engine& e) {
        e.rtm_shots(e.range_s0(), e.range_n(), data_all + e.survey_offset(e.range_s0()), false);
    });
}

int fwi_rtm_survey_dev(fwi_ctx* ctx, const float* d_data_all) {
    if (!d_data_all) return arg_error(ctx, "NULL data");
    return guarded(ctx, [&](fwi::Engine& e) {
        e.rtm_shots(e.range_s0(), e.range_n(), d_data_all + e.survey_offset(e.range_s0()), true);
    });
}

int fwi_rtm_image(fwi_ctx* ctx, float* image) {
    if (!image) return arg_error(ctx, "NULL image");
    return guarded(ctx, [&](fwi::Engine& e) { e.rtm_image(image); });
}

int fwi_rtm_raw(fwi_ctx* ctx, float* image, float* illum) {
    return guarded(ctx, [&](fwi::Engine& e) { e.rtm_raw(image, illum); });
}

int fwi_set_observed(fwi_ctx* ctx, const float* obs_all) {
    if (!obs_all) return arg_error(ctx, "NULL observed data");
    return guarded(ctx, [&](fwi::Engine& e) { e.set_observed(obs_all, false); });
}

int fwi_set_observed_dev(fwi_ctx* ctx, const float* d_obs_all) {
    if (!d_obs_all) return arg_error(ctx, "NULL observed data");
    return guarded(ctx, [&](fwi::Engine& e) { e.set_observed(d_obs_all, true); });
}

int fwi_compute_gradient(fwi_ctx* ctx, int with_gradient, double* sum_res) {
    return guarded(ctx, [&](fwi::Engine& e) {
        double s = e.compute_gradient(with_gradient != 0);
        if (sum_res) *sum_res = s;
    });
}

int fwi_set_shot_range(fwi_ctx* ctx, int s0, int ns) {
    return guarded(ctx, [&](fwi::Engine& e) { e.set_shot_range(s0, ns); });
}

int fwi_gradient_accumulate(fwi_ctx* ctx, int with_gradient, double* sum_res) {
    return guarded(ctx, [&](fwi::Engine& e) {
        double s = e.accumulate_gradient(with_gradient != 0);
        if (sum_res) *sum_res = s;
    });
}

int fwi_gradient_finish(fwi_ctx* ctx) {
    return guarded(ctx, [&](fwi::Engine& e) { e.finish_gradient(); });
}

int fwi_accumulators(fwi_ctx* ctx, float** a, float** b) {
    if (!a || !b) return arg_error(ctx, "NULL output");
    return guarded(ctx, [&](fwi::Engine& e) {
        e.accumulators(a, b);
        e.stream_sync();
    });
}

int fwi_trial_steps(fwi_ctx* ctx, float* a1, float* a2) {
    if (!a1 || !a2) return arg_error(ctx, "NULL output");
    return guarded(ctx, [&](fwi::Engine& e) { e.trial_steps(a1, a2); });
}

int fwi_parabola_step(fwi_ctx* ctx, float f0, float f1, float f2, float* step) {
    if (!step) return arg_error(ctx, "NULL step");
    return guarded(ctx, [&](fwi::Engine& e) { *step = e.parabola_step(f0, f1, f2); });
}

int fwi_set_direction(fwi_ctx* ctx, const float* dir) {
    return guarded(ctx, [&](fwi::Engine& e) { e.set_direction(dir, false); });
}

int fwi_set_direction_dev(fwi_ctx* ctx, const float* d_dir) {
    return guarded(ctx, [&](fwi::Engine& e) { e.set_direction(d_dir, true); });
}

int fwi_get_gradient(fwi_ctx* ctx, float* g) {
    if (!g) return arg_error(ctx, "NULL gradient");
    return guarded(ctx, [&](fwi::Engine& e) { e.get_gradient(g); });
}

int fwi_get_gradient_raw(fwi_ctx* ctx, float* g, float* illum) {
    return guarded(ctx, [&](fwi::Engine& e) { e.get_gradient_raw(g, illum); });
}

int fwi_linesearch_trial(fwi_ctx* ctx, float alpha, double* sum_res) {
    return guarded(ctx, [&](fwi::Engine& e) {
        double s = e.linesearch_trial(alpha);
        if (sum_res) *sum_res = s;
    });
}

int fwi_optimization(fwi_ctx* ctx, float f0, float* step) {
    if (!step) return arg_error(ctx, "NULL step");
    return guarded(ctx, [&](fwi::Engine& e) { *step = e.optimization(f0); });
}

int fwi_update_model(fwi_ctx* ctx, float step, float* vp_out) {
    return guarded(ctx, [&](fwi::Engine& e) { e.update_model(step, vp_out); });
}

int fwi_mute_direct(fwi_ctx* ctx, float* data_all, float velocity, float delay, float gstd) {
    return guarded(ctx, [&](fwi::Engine& e) { e.mute_direct(data_all, false, velocity, delay, gstd); });
}

int fwi_mute_direct_dev(fwi_ctx* ctx, float* d_data_all, float velocity, float delay, float gstd) {
    return guarded(ctx, [&](fwi::Engine& e) { e.mute_direct(d_data_all, true, velocity, delay, gstd); });
}

int fwi_smooth_model(fwi_ctx* ctx, const float* vp, float sigma, float depth_mask, float* vp_out) {
    return guarded(ctx, [&](fwi::Engine& e) { e.smooth_model(vp, sigma, depth_mask, vp_out); });
}

int fwi_update_model_bounded(fwi_ctx* ctx, float step, float vmin, float vmax, float* vp_out) {
    return guarded(ctx, [&](fwi::Engine& e) { e.update_model(step, vp_out, vmin, vmax); });
}

int fwi_random_boundary(fwi_ctx* ctx, int shot, float* vp_rbc) {
    if (!vp_rbc) return arg_error(ctx, "NULL output");
    return guarded(ctx, [&](fwi::Engine& e) { e.random_boundary(shot, vp_rbc); });
}

int fwi_util_parameter(const char* params_path, const char* key, char* buf, size_t len) {
    if (!params_path || !key || !buf) return FWI_ERR_ARG;
    try {
        fwi::ParamFile p(params_path);
        std::string v = p.str(key);
        if (v.size() + 1 > len) return FWI_ERR_ARG;
        std::memcpy(buf, v.c_str(), v.size() + 1);
        return FWI_OK;
    } catch (const fwi::Error& e) {
        return e.code;
    }
}

int fwi_util_wavelet(int nt, float dt, float fmax, float* out, int* tlag) {
    if (!out || !tlag || nt <= 0) return FWI_ERR_ARG;
    try {
        std::vector<float> w = fwi::make_wavelet(nt, dt, fmax, tlag);
        std::memcpy(out, w.data(), w.size() * sizeof(float));
        return FWI_OK;
    } catch (const fwi::Error& e) {
        return e.code;
    }
}

int fwi_util_b1d(int nb, float abc_factor, float* out) {
    if (!out || nb <= 0) return FWI_ERR_ARG;
    std::vector<float> b = fwi::make_b1d(nb, abc_factor);
    std::memcpy(out, b.data(), b.size() * sizeof(float));
    return FWI_OK;
}

int fwi_util_grid_index(int n, const float* coord, float dh, int nb, int* out) {
    if (!coord || !out || n < 0) return FWI_ERR_ARG;
    for (int k = 0; k < n; ++k) out[k] = fwi::grid_index(coord[k], dh, nb);
    return FWI_OK;
}

int fwi_util_bumps(int nxx, int nzz, int nb, float dh, float ratio, float varVp, uint64_t seed, uint32_t shot,
                   float* out, int cap, int* count) {
    if (!count || (cap > 0 && !out) || !(ratio > 0) || nxx < 2 || nzz < 2) return FWI_ERR_ARG;
    std::vector<fwi::Bump> b = fwi::make_bumps(nxx, nzz, nb, dh, ratio, varVp, seed, shot);
    *count = (int)b.size();
    for (int k = 0; k < (int)b.size() && k < cap; ++k) {
        float* o = out + 5 * (size_t)k;
        o[0] = b[k].xc;
        o[1] = b[k].zc;
        o[2] = b[k].r;
        o[3] = b[k].A;
        o[4] = b[k].factor;
    }
    return FWI_OK;
}

int fwi_util_window(float xs, float max_offset, int nx, float dh, int* c0, int* w) {
    if (!c0 || !w || nx < 9 || !(dh > 0)) return FWI_ERR_ARG;
    try {
        fwi::Geometry g;
        g.xsrc = {xs};
        g.zsrc = {0.0f};
        const auto win = fwi::aperture_windows(g, nx, dh, {max_offset});
        *c0 = win[0].c0;
        *w = win[0].w;
        return FWI_OK;
    } catch (const fwi::Error& e) {
        g_create_error = e.what();
        return e.code;
    }
}

int fwi_util_normal(uint64_t seed, uint32_t shot, uint32_t stream, uint64_t ctr, float* out) {
    if (!out) return FWI_ERR_ARG;
    *out = detm::normalf(detm::stream_key(seed, shot, stream), ctr);
    return FWI_OK;
}

int fwi_residual_noalloc(const float* d_obs, const float* d_cal, float* d_res, size_t n, double* d_sum,
                         void* stream) {
    std::string err;
    int rc = fwi::residual_noalloc(d_obs, d_cal, d_res, n, d_sum, static_cast<cudaStream_t>(stream), &err);
    if (rc != FWI_OK) g_create_error = err;
    else g_create_error.clear();  // no stale message after a call that succeeded
    return rc;
}

int fwi_describe(fwi_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !ctx->eng || !buf || len == 0) return FWI_ERR_ARG;
    std::string s = ctx->eng->last_fwd_plan;
    if (!ctx->eng->last_bwd_plan.empty()) s += " || backward: " + ctx->eng->last_bwd_plan;
    if (s.size() + 1 > len) return FWI_ERR_ARG;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return FWI_OK;
}

int fwi_launch_count(fwi_ctx* ctx, long long* count, int reset) {
    if (!count) return arg_error(ctx, "NULL count");
    return guarded(ctx, [&](fwi::Engine& e) { *count = e.launches(reset != 0); });
}

int fwi_fwd_timing(fwi_ctx* ctx, int enable) {
    return guarded(ctx, [&](fwi::Engine& e) { e.fwd_timing(enable != 0); });
}

int fwi_fwd_timing_read(fwi_ctx* ctx, double* ms, long long* launches, long long* updates) {
    if (!ms || !launches || !updates) return arg_error(ctx, "NULL output");
    return guarded(ctx, [&](fwi::Engine& e) { e.fwd_timing_read(ms, launches, updates); });
}

int fwi_bwd_timing_read(fwi_ctx* ctx, double* ms, long long* launches, long long* updates) {
    if (!ms || !launches || !updates) return arg_error(ctx, "NULL output");
    return guarded(ctx, [&](fwi::Engine& e) { e.bwd_timing_read(ms, launches, updates); });
}

}  // extern "C"
