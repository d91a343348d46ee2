// app_common.hpp — helpers shared by the three drop-in executables.
#pragma once
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/fwi2d.h"

namespace app {

inline int fail(fwi_ctx* ctx, const char* what) {
    std::fprintf(stderr, "Error: %s: %s\n", what, fwi_last_error(ctx));
    if (ctx) fwi_ctx_destroy(ctx);
    return 1;
}

inline bool param(fwi_ctx* ctx, const char* key, std::string* out) {
    std::vector<char> buf(4096);
    if (fwi_get_param(ctx, key, buf.data(), buf.size()) != FWI_OK) return false;
    *out = buf.data();
    return true;
}

inline bool read_floats(const std::string& path, float* dst, size_t n) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) {
        std::fprintf(stderr, "Error: %s could not be opened!\n", path.c_str());
        return false;
    }
    f.read(reinterpret_cast<char*>(dst), (std::streamsize)(n * sizeof(float)));
    if ((size_t)f.gcount() != n * sizeof(float)) {
        std::fprintf(stderr, "Error: %s holds fewer than %zu float32 values\n", path.c_str(), n);
        return false;
    }
    return true;
}

inline bool write_floats(const std::string& path, const float* src, size_t n, bool announce = true) {
    std::ofstream f(path, std::ios::binary);
    if (!f.is_open()) {
        std::fprintf(stderr, "Error: %s could not be opened!\n", path.c_str());
        return false;
    }
    f.write(reinterpret_cast<const char*>(src), (std::streamsize)(n * sizeof(float)));
    if (announce) std::printf("\nBinary file %s was successfully written.\n", path.c_str());
    return (bool)f;
}

// Per-shot file I/O on a small pool of host threads (the reference reads and
// writes one shot at a time, inversion.cu:168-172, modeling.cu:279-284): runs
// fn(i) for i in [0, n) and returns whether every call succeeded.
template <class F>
bool parallel_files(int n, F fn) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int workers = std::max(1, std::min(n, (int)std::min(16u, hw)));
    std::atomic<int> next{0};
    std::atomic<bool> ok{true};
    std::vector<std::thread> pool;
    pool.reserve(workers);
    for (int t = 0; t < workers; ++t)
        pool.emplace_back([&] {
            for (int i = next++; i < n; i = next++)
                if (!fn(i)) ok = false;
        });
    for (auto& th : pool) th.join();
    return ok;
}

inline std::string banner(const char* title) {
    std::string line(80, '-');
    return line + "\n" + std::string((80 - std::string(title).size()) / 2, ' ') + title + "\n" + line + "\n";
}

using clock = std::chrono::system_clock;
inline double seconds(clock::time_point a, clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

}  // namespace app
