// migration — drop-in for src/migration_main.cpp: reverse-time migration of
// every shot through a random boundary, then the RTM section file of
// Migration::export_seismic (src/migration/migration.cu:90-115).
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
    if (fwi_ctx_create(argv[1], FWI_MODE_MIGRATION, &ctx) != FWI_OK) return app::fail(nullptr, "set_parameters");
    fwi_dims d;
    fwi_get_dims(ctx, &d);
    std::string in_folder, in_prefix, out_folder;
    if (!app::param(ctx, "mig_input_folder", &in_folder)) return app::fail(ctx, "mig_input_folder");
    if (!app::param(ctx, "mig_input_prefix", &in_prefix)) return app::fail(ctx, "mig_input_prefix");
    if (!app::param(ctx, "mig_output_folder", &out_folder)) return app::fail(ctx, "mig_output_folder");
    std::printf("%s", app::banner("Reverse Time Migration").c_str());
    std::printf("Model dimensions: (z = %g, x = %g) m\n\n", (d.nz - 1) * d.dh, (d.nx - 1) * d.dh);

    const size_t per = (size_t)d.nt * d.nrec;
    std::vector<float> data(per * d.nsrc);
    // set_seismic_source, migration.cu:83-88
    if (!app::parallel_files(d.nsrc, [&](int s) {
            return app::read_floats(in_folder + in_prefix + std::to_string(s + 1) + ".bin", data.data() + per * s, per);
        })) {
        fwi_ctx_destroy(ctx);
        return 1;
    }
    auto ti = app::clock::now();
    if (fwi_rtm_survey(ctx, data.data()) != FWI_OK) return app::fail(ctx, "migration");
    auto tf = app::clock::now();
    std::vector<float> image((size_t)d.nx * d.nz);
    if (fwi_rtm_image(ctx, image.data()) != FWI_OK) return app::fail(ctx, "export_seismic");
    char dh[32], fm[32];
    std::snprintf(dh, sizeof dh, "%d", (int)d.dh);
    std::snprintf(fm, sizeof fm, "%d", (int)d.fmax);
    std::string file = out_folder + "RTM_section_" + fm + "Hz_" + std::to_string(d.nz) + "x" + std::to_string(d.nx) +
                       "_" + dh + "m.bin";
    if (!app::write_floats(file, image.data(), image.size())) return app::fail(ctx, "export_seismic");
    std::printf("\nRun time: %g s.\n", app::seconds(ti, tf));
    fwi_ctx_destroy(ctx);
    return 0;
}
