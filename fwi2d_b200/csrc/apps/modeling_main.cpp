// modeling — drop-in for src/modeling_main.cpp: models every shot of the
// survey described by parameters.txt and writes one seismogram file per shot
// (names and layout of Modeling::get_seismogram, src/modeling/modeling.cu:279-284).
// All shots run batched on the GPU; files are written afterwards.
#include <cstdio>
#include <string>
#include <vector>

#include "app_common.hpp"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s parameters.txt\n", argv[0]);
        return 2;
    }
    fwi_ctx* ctx = nullptr;
    if (fwi_ctx_create(argv[1], FWI_MODE_MODELING, &ctx) != FWI_OK) return app::fail(nullptr, "set_parameters");
    fwi_dims d;
    fwi_get_dims(ctx, &d);
    std::string folder;
    if (!app::param(ctx, "mod_output_folder", &folder)) return app::fail(ctx, "mod_output_folder");
    std::printf("%s", app::banner("Seismic Modeling").c_str());
    std::printf("Model dimensions: (z = %g, x = %g) m\n\n", (d.nz - 1) * d.dh, (d.nx - 1) * d.dh);
    std::printf("Running %d shots in batches on the GPU\n\n", d.nsrc);

    const size_t per = (size_t)d.nt * d.nrec;
    std::vector<float> seis(per * d.nsrc);
    auto ti = app::clock::now();
    if (fwi_model_survey(ctx, seis.data()) != FWI_OK) return app::fail(ctx, "forward_solver");
    char us[64];
    std::snprintf(us, sizeof us, "%d", int(1e6f * d.dt));
    auto file_of = [&](int s) {
        return folder + "seismogram_nt" + std::to_string(d.nt) + "_nr" + std::to_string(d.nrec) + "_" + us +
               "us_shot_" + std::to_string(s + 1) + ".bin";
    };
    // get_seismogram for every shot, the files written by a thread pool
    if (!app::parallel_files(d.nsrc,
                             [&](int s) { return app::write_floats(file_of(s), seis.data() + per * s, per, false); }))
        return app::fail(ctx, "get_seismogram");
    for (int s = 0; s < d.nsrc; ++s) std::printf("\nBinary file %s was successfully written.\n", file_of(s).c_str());
    auto tf = app::clock::now();
    std::printf("\nRun time: %g s.\n", app::seconds(ti, tf));
    fwi_ctx_destroy(ctx);
    return 0;
}
