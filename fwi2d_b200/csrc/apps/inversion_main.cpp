// inversion — drop-in for src/inversion_main.cpp: L2 full-waveform inversion
// with the parabolic line search of Inversion::optimization, writing the model
// of every iteration, the convergence curve and the final model under the
// reference's names (src/inversion/inversion.cu:344-379).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "app_common.hpp"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s parameters.txt\n", argv[0]);
        return 2;
    }
    fwi_ctx* ctx = nullptr;
    if (fwi_ctx_create(argv[1], FWI_MODE_INVERSION, &ctx) != FWI_OK) return app::fail(nullptr, "set_parameters");
    fwi_dims d;
    fwi_get_dims(ctx, &d);
    std::string in_folder, in_prefix, out_folder, res_folder, max_it_s;
    if (!app::param(ctx, "inv_input_folder", &in_folder)) return app::fail(ctx, "inv_input_folder");
    if (!app::param(ctx, "inv_input_prefix", &in_prefix)) return app::fail(ctx, "inv_input_prefix");
    if (!app::param(ctx, "inv_output_folder", &out_folder)) return app::fail(ctx, "inv_output_folder");
    if (!app::param(ctx, "inv_residuo_folder", &res_folder)) return app::fail(ctx, "inv_residuo_folder");
    if (!app::param(ctx, "max_iteration", &max_it_s)) return app::fail(ctx, "max_iteration");
    const int max_iteration = std::stoi(max_it_s);
    std::printf("%s", app::banner("Full Waveform Inversion").c_str());

    const size_t per = (size_t)d.nt * d.nrec;
    std::vector<float> obs(per * d.nsrc);
    // set_obs_data, inversion.cu:168-172: every shot's file, read in parallel
    if (!app::parallel_files(d.nsrc, [&](int s) {
            return app::read_floats(in_folder + in_prefix + std::to_string(s + 1) + ".bin", obs.data() + per * s, per);
        })) {
        fwi_ctx_destroy(ctx);
        return 1;
    }
    if (fwi_set_observed(ctx, obs.data()) != FWI_OK) return app::fail(ctx, "set_obs_data");

    char fm[32], dh[32];
    std::snprintf(fm, sizeof fm, "%d", (int)d.fmax);
    std::snprintf(dh, sizeof dh, "%d", (int)d.dh);
    const std::string suffix = std::string(fm) + "Hz_" + std::to_string(d.nz) + "x" + std::to_string(d.nx) + "_" + dh + "m.bin";
    std::vector<float> vp((size_t)d.nx * d.nz);
    std::vector<float> residuo;
    auto ti = app::clock::now();
    for (int it = 0; it <= max_iteration; ++it) {
        double sum_res = 0.0;
        // the last pass only measures the residual (inversion.cu:117, 136)
        if (fwi_compute_gradient(ctx, it < max_iteration, &sum_res) != FWI_OK) return app::fail(ctx, "compute_gradient");
        residuo.push_back(std::sqrt((float)sum_res));
        if (it == 0) std::printf("-------- Computing first residuo --------\n");
        std::printf("Iteration %d of %d, residuo: %g\n", it, max_iteration, residuo.back());
        if (it == max_iteration) break;
        float step = 0.0f;
        if (fwi_optimization(ctx, residuo.back(), &step) != FWI_OK) return app::fail(ctx, "optimization");
        if (fwi_update_model(ctx, step, vp.data()) != FWI_OK) return app::fail(ctx, "update_model");
        std::string file = out_folder + "model_FWI_iteration_" + std::to_string(it + 1) + "_" + suffix;
        if (!app::write_floats(file, vp.data(), vp.size())) return app::fail(ctx, "update_model");
    }
    std::printf("Final residuo: %g\n\n", residuo.back());
    // export_convergence, inversion.cu:360-372
    std::string conv = res_folder + "convergence_" + std::to_string(max_iteration) + "_iterations.txt";
    std::ofstream rf(conv);
    if (!rf.is_open()) return app::fail(ctx, "export_convergence");
    for (int r = 0; r <= max_iteration; ++r) rf << residuo[r] << "\n";
    rf.close();
    std::printf("Text file %s was successfully written.\n", conv.c_str());
    // export_final_model, inversion.cu:374-379
    if (fwi_get_model(ctx, vp.data()) != FWI_OK) return app::fail(ctx, "export_final_model");
    if (!app::write_floats(out_folder + "final_model_FWI_" + suffix, vp.data(), vp.size()))
        return app::fail(ctx, "export_final_model");
    auto tf = app::clock::now();
    std::printf("\nRun time: %g s.\n", app::seconds(ti, tf));
    fwi_ctx_destroy(ctx);
    return 0;
}
