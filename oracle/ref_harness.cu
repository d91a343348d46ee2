// ref_harness.cu — drives the reference's own CUDA code to produce golden
// vectors (TEST INFRASTRUCTURE; built by `make -C oracle ref` into oracle/_ref).
//
// It links the reference sources where they lie (src/admin, src/geometry,
// src/modeling, src/migration, src/inversion) and, through a subclass of the
// reference's Modeling class, runs:
//   * set_parameters (wavelet through FFTW -> cuFFTW, ABC tables, model, geometry)
//   * per shot: initialization + forward_solver (compute_pressure +
//     compute_seismogram), dumping the seismogram and the final two fields;
//   * optionally the backward loops of Migration::backward_propagation
//     (inject_seismogram + cross_correlation, migration.cu:61-81) and of
//     Inversion::backward_propagation (inject_adjoint + build_gradient,
//     inversion.cu:230-248) on a forward run without ABC, for a given padded
//     velocity and given input traces.
// The reference's random-boundary kernels are NOT called: random_boundary_bg
// and random_boundary_gp index past the end of Vp and X for the threads of the
// last block (modeling.cu:467-524), so the harness takes the boundary velocity
// as an input file instead.
//
// usage: ref_harness <parameters.txt> <outdir> [vel_padded.bin data_prefix]
//   without the optional arguments: ABC modeling of every shot;
//   with them: ABC off, d_Vp replaced by vel_padded.bin (nzz x nxx), then per
//   shot forward + RTM backward and forward + gradient backward, with the input
//   traces of shot k read from <data_prefix><k>.bin.
// usage: ref_harness --time <parameters.txt> <vel_padded.bin> <data_prefix> <reps>
//   times, with CUDA events on the default stream, the reference's own loops
//   on every shot: forward_solver (compute_pressure + compute_seismogram,
//   modeling.cu:286-299, ABC off), the migration back-propagation
//   (inject_seismogram + cross_correlation, migration.cu:61-81) and the
//   adjoint back-propagation (inject_adjoint + build_gradient,
//   inversion.cu:230-248); prints one line per repetition:
//   "time fwd_ms=... rtm_bwd_ms=... grad_bwd_ms=... fwd_abc_ms=... updates=..."
//   (fwd_abc: forward_solver with the absorbing boundary on, the modeling's
//   propagation) where updates = shots x nxx x nzz x (nt + tlag) per
//   propagation.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "inversion/inversion.cuh"
#include "migration/migration.cuh"
#include "modeling/modeling.cuh"

static void save(const std::string& path, const float* d_ptr, size_t n) {
    std::vector<float> h(n);
    cudaMemcpy(h.data(), d_ptr, n * sizeof(float), cudaMemcpyDeviceToHost);
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { std::fprintf(stderr, "cannot write %s\n", path.c_str()); std::exit(2); }
    std::fwrite(h.data(), sizeof(float), n, f);
    std::fclose(f);
}

static std::vector<float> load(const std::string& path, size_t n) {
    std::vector<float> h(n);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(h.data(), sizeof(float), n, f) != n) { std::fprintf(stderr, "cannot read %s\n", path.c_str()); std::exit(2); }
    std::fclose(f);
    return h;
}

// The source injection of compute_pressure (modeling.cu:316-317) is an
// atomicAdd by global thread 0 that races with the stencil reads of P and with
// the owner's in-place `P[index] *= damper` (modeling.cu:341), which can write
// back the pre-injection value.  When every block of a step is resident at
// once (all grids here, and the reference configurations on a 148-SM B200)
// the outcome differs from step to step and shot to shot.  The harness
// therefore injects in a launch of its own before compute_pressure and calls
// compute_pressure with nt = 0, which switches its own injection off and
// leaves the rest of the kernel unchanged.
__global__ void harness_add_source(float* P, int idx, float idh2, const float* wavelet, int t) {
    P[idx] += idh2 * wavelet[t];
}

class Driver : public Modeling {
public:
    // forward_solver (modeling.cu:286-299) with the injection in its own launch
    void forward_solver_ordered() {
        cudaMemset(d_P, 0, matsize * sizeof(float));
        cudaMemset(d_Pold, 0, matsize * sizeof(float));
        for (int tId = 0; tId < nt + tlag; tId++) {
            if (tId < nt) harness_add_source<<<1, 1>>>(d_P, sIdz + sIdx * nzz, idh2, d_wavelet, tId);
            compute_pressure<<<nBlocks, NTHREADS>>>(d_Vp, d_P, d_Pold, d_wavelet, d_b1d, d_b2d, sIdx, sIdz, tId, 0,
                                                    nb, nxx, nzz, idh2, dt, ABC);
            compute_seismogram<<<sBlocks, NTHREADS>>>(d_P, d_rIdx, d_rIdz, d_seismogram, geometry->nrec, tId, tlag, nt,
                                                      nzz);
            std::swap(d_P, d_Pold);
        }
    }

    // one back-propagation of the current source field, as the reference's loops
    void backward_loop(int mode, float* d_Pr, float* d_Prold, float* d_acc, float* d_ill) {
        const int nrec = geometry->nrec;
        for (int tId = 0; tId < nt + tlag; tId++) {
            if (mode == 0) {
                inject_seismogram<<<sBlocks, NTHREADS>>>(d_Pr, d_rIdx, d_rIdz, d_seismogram, nrec, tId, nt, nzz, idh2);
                cross_correlation<<<nBlocks, NTHREADS>>>(d_P, d_Pold, d_Pr, d_Prold, d_Vp, d_acc, d_ill, nxx, nzz, idh2, dt);
            } else {
                inject_adjoint<<<sBlocks, NTHREADS>>>(d_Pr, d_rIdx, d_rIdz, d_seismogram, nrec, tId, nt, nzz, idh2);
                build_gradient<<<nBlocks, NTHREADS>>>(d_P, d_Pold, d_Pr, d_Prold, d_Vp, d_acc, d_ill, nxx, nzz, nt, dt, idh2);
            }
            std::swap(d_P, d_Pold);
            std::swap(d_Pr, d_Prold);
        }
    }

    void time_loops(const std::string& params, const char* vel_file, const char* data_prefix, int reps) {
        parameters = params;
        set_parameters();
        ABC = false;
        const int nrec = geometry->nrec;
        std::vector<float> v = load(vel_file, (size_t)matsize);
        cudaMemcpy(d_Vp, v.data(), matsize * sizeof(float), cudaMemcpyHostToDevice);
        float *d_Pr = nullptr, *d_Prold = nullptr, *d_acc = nullptr, *d_ill = nullptr;
        cudaMalloc(&d_Pr, matsize * sizeof(float));
        cudaMalloc(&d_Prold, matsize * sizeof(float));
        cudaMalloc(&d_acc, matsize * sizeof(float));
        cudaMalloc(&d_ill, matsize * sizeof(float));
        std::vector<std::vector<float>> data(geometry->nsrc);
        for (int s = 0; s < geometry->nsrc; ++s)
            data[s] = load(std::string(data_prefix) + std::to_string(s + 1) + ".bin", (size_t)nt * nrec);
        cudaEvent_t e[2];
        cudaEventCreate(&e[0]);
        cudaEventCreate(&e[1]);
        auto timed = [&](auto&& fn) {
            cudaEventRecord(e[0]);
            fn();
            cudaEventRecord(e[1]);
            cudaEventSynchronize(e[1]);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e[0], e[1]);
            return (double)ms;
        };
        for (int r = 0; r < reps; ++r) {
            double fwd = 0, rtm = 0, grad = 0, fwd_abc = 0;
            for (srcId = 0; srcId < geometry->nsrc; srcId++) {
                initialization();
                ABC = true;  // the modeling's propagation (absorbing boundary on)
                fwd_abc += timed([&] { forward_solver(); });
                ABC = false;
                for (int mode = 0; mode < 2; ++mode) {
                    fwd += timed([&] { forward_solver(); });
                    cudaMemcpy(d_seismogram, data[srcId].data(), data[srcId].size() * sizeof(float),
                               cudaMemcpyHostToDevice);
                    cudaMemset(d_Pr, 0, matsize * sizeof(float));
                    cudaMemset(d_Prold, 0, matsize * sizeof(float));
                    cudaMemset(d_acc, 0, matsize * sizeof(float));
                    cudaMemset(d_ill, 0, matsize * sizeof(float));
                    (mode == 0 ? rtm : grad) += timed([&] { backward_loop(mode, d_Pr, d_Prold, d_acc, d_ill); });
                }
            }
            cudaError_t err = cudaDeviceSynchronize();
            if (err != cudaSuccess) { std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err)); std::exit(3); }
            std::printf("time fwd_ms=%.4f rtm_bwd_ms=%.4f grad_bwd_ms=%.4f fwd_abc_ms=%.4f updates=%lld\n", fwd / 2,
                        rtm, grad, fwd_abc, (long long)geometry->nsrc * nxx * nzz * (nt + tlag));
            std::fflush(stdout);
        }
    }

    void run(const std::string& params, const std::string& out, const char* vel_file, const char* data_prefix) {
        parameters = params;
        set_parameters();
        save(out + "/wavelet.bin", d_wavelet, nt);
        save(out + "/b1d.bin", d_b1d, nb);
        const int nrec = geometry->nrec;
        if (vel_file) {
            ABC = false;
            std::vector<float> v = load(vel_file, (size_t)matsize);
            cudaMemcpy(d_Vp, v.data(), matsize * sizeof(float), cudaMemcpyHostToDevice);
        }
        float *d_Pr = nullptr, *d_Prold = nullptr, *d_acc = nullptr, *d_ill = nullptr;
        if (vel_file) {
            cudaMalloc(&d_Pr, matsize * sizeof(float));
            cudaMalloc(&d_Prold, matsize * sizeof(float));
            cudaMalloc(&d_acc, matsize * sizeof(float));
            cudaMalloc(&d_ill, matsize * sizeof(float));
        }
        for (srcId = 0; srcId < geometry->nsrc; srcId++) {
            initialization();
            const std::string k = std::to_string(srcId + 1);
            cudaMemset(d_seismogram, 0, (size_t)nt * nrec * sizeof(float));
            forward_solver();  // as the reference runs it, injection race included
            save(out + "/seis_raw_" + k + ".bin", d_seismogram, (size_t)nt * nrec);
            cudaMemset(d_seismogram, 0, (size_t)nt * nrec * sizeof(float));
            forward_solver_ordered();
            save(out + "/seis_" + k + ".bin", d_seismogram, (size_t)nt * nrec);
            save(out + "/p_" + k + ".bin", d_P, matsize);
            save(out + "/pold_" + k + ".bin", d_Pold, matsize);
            if (!vel_file) continue;
            std::vector<float> data = load(std::string(data_prefix) + k + ".bin", (size_t)nt * nrec);
            for (int mode = 0; mode < 2; ++mode) {
                if (mode == 1) forward_solver_ordered();  // fresh source field for the gradient pass
                cudaMemcpy(d_seismogram, data.data(), data.size() * sizeof(float), cudaMemcpyHostToDevice);
                cudaMemset(d_Pr, 0, matsize * sizeof(float));
                cudaMemset(d_Prold, 0, matsize * sizeof(float));
                cudaMemset(d_acc, 0, matsize * sizeof(float));
                cudaMemset(d_ill, 0, matsize * sizeof(float));
                backward_loop(mode, d_Pr, d_Prold, d_acc, d_ill);
                const char* tag = mode == 0 ? "image" : "grad";
                save(out + "/" + tag + "_" + k + ".bin", d_acc, matsize);
                save(out + "/" + tag + "_illum_" + k + ".bin", d_ill, matsize);
            }
        }
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) { std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e)); std::exit(3); }
        std::printf("nb=%d nxx=%d nzz=%d tlag=%d nt=%d nrec=%d\n", nb, nxx, nzz, tlag, nt, nrec);
    }
};

int main(int argc, char** argv) {
    if (argc == 6 && std::string(argv[1]) == "--time") {
        Driver d;
        d.time_loops(argv[2], argv[3], argv[4], std::atoi(argv[5]));
        return 0;
    }
    if (argc != 3 && argc != 5) {
        std::fprintf(stderr, "usage: %s parameters.txt outdir [vel_padded.bin data_prefix]\n", argv[0]);
        return 1;
    }
    Driver d;
    d.run(argv[1], argv[2], argc == 5 ? argv[3] : nullptr, argc == 5 ? argv[4] : nullptr);
    return 0;
}
