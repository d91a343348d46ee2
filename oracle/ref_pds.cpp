// ref_pds.cpp — runs the reference's own host-side Poisson-disk sampler
// (poissonDiskSampling, src/admin/admin.cpp:115-206) with a fixed seed
// (TEST INFRASTRUCTURE; built by `make -C oracle ref` into oracle/_ref).
//
// The reference draws from a global std::mt19937 `rng` seeded by
// std::random_device (admin.cpp:112-113), so its point sets cannot be
// reproduced from run to run.  The generator has external linkage: this
// harness reseeds it before each call, which leaves the sampler unchanged and
// makes its output a function of the seed, so the statistics of its point
// sets can be compared with this project's counter-based sampler.
//
// usage: ref_pds <seed> <x_max> <z_max> <radius>
//   prints one "x z" line per point, in the sampler's order.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "admin/admin.hpp"

extern std::mt19937 rng;

int main(int argc, char** argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s seed x_max z_max radius\n", argv[0]);
        return 1;
    }
    rng.seed((std::mt19937::result_type)std::strtoul(argv[1], nullptr, 10));
    const std::vector<Point> pts =
        poissonDiskSampling(std::strtof(argv[2], nullptr), std::strtof(argv[3], nullptr), std::strtof(argv[4], nullptr));
    for (const Point& p : pts) std::printf("%.9g %.9g\n", p.x, p.z);
    return 0;
}
