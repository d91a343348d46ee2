// k_noalloc.cu — residual and FP64 misfit without any device allocation.
//
// Some callers cannot call cudaMalloc: a host application that owns and
// reserves all device memory through its own pool (a framework's caching
// allocator, a plugin host), code that runs inside a CUDA stream capture where
// an allocation would break the capture, and processing loops where the
// implicit device synchronisation of cudaMalloc is not acceptable.  For them
// this file computes res = obs - cal and sum(res^2) with its only scratch - the
// per-chunk partial sums - in a file-scope __device__ array, so the call
// allocates nothing.  The caller passes every input and output as device
// memory and a stream; the call only enqueues work.
//
// The array is a host-side stand-in in host code: its device address is looked
// up with cudaGetSymbolAddress once per device (with that device current) on
// the first call made on that device, and only that address is passed to the
// kernels.  Every GPU that loads the library holds the array (64 KiB) until
// the process exits.  All calls share it and it keeps the contents of the last
// call, so calls that overlap on the GPU (different streams, or other host
// threads) race with each other; serialise them.  Each call overwrites every
// partial it later reads, so nothing has to be cleared between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "kernels.h"

namespace fwi {

namespace {

constexpr int kChunk = 8192;             // samples reduced into one partial sum
constexpr int kMaxPartials = 8192;       // scratch: 8192 partials + 1 result slot
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kMaxPartials + 1];

// One block per chunk; the block sums its chunk in a fixed order, so the
// result depends only on n, not on the GPU.
__global__ void residual_chunk_kernel(const float* __restrict__ obs, const float* __restrict__ cal,
                                      float* __restrict__ res, size_t n, double* __restrict__ partial) {
    __shared__ double red[kThreads / 32];
    const size_t base = (size_t)blockIdx.x * kChunk;
    const size_t end = base + kChunk < n ? base + kChunk : n;
    double acc = 0.0;
    for (size_t c = base + threadIdx.x; c < end; c += kThreads) {
        const float r = obs[c] - cal[c];
        res[c] = r;
        acc += (double)r * (double)r;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += red[w];
        partial[blockIdx.x] = t;
    }
}

__global__ void sum_chunks_kernel(const double* __restrict__ partial, int count, double* out_scratch,
                                  double* out) {
    __shared__ double red[kThreads / 32];
    double acc = 0.0;
    for (int c = threadIdx.x; c < count; c += kThreads) acc += partial[c];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += red[w];
        *out_scratch = t;
        *out = t;
    }
}

std::mutex g_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once).
cudaError_t scratch_address(double** out, std::string* err) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return e;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        *err = "device ordinal out of range for the no-allocation scratch table";
        return cudaErrorInvalidDevice;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            *err = std::string("cudaGetSymbolAddress of the no-allocation scratch: ") + cudaGetErrorString(e);
            return e;
        }
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace

size_t noalloc_max_samples() { return (size_t)kChunk * kMaxPartials; }

// Returns 0 or a negative FWI_ERR_* code (-8 argument, -3 CUDA) with *err set.
int residual_noalloc(const float* d_obs, const float* d_cal, float* d_res, size_t n, double* d_sum,
                     cudaStream_t st, std::string* err) {
    if (!d_obs || !d_cal || !d_res || !d_sum) {
        *err = "fwi_residual_noalloc: NULL device pointer";
        return -8;
    }
    if (n > noalloc_max_samples()) {
        *err = "fwi_residual_noalloc: n = " + std::to_string(n) + " samples exceeds the maximum of " +
               std::to_string(noalloc_max_samples()) + " (8192 partial sums of 8192 samples); split the call";
        return -8;
    }
    double* scratch = nullptr;
    if (scratch_address(&scratch, err) != cudaSuccess) return -3;
    const int chunks = (int)((n + kChunk - 1) / kChunk);
    if (chunks > 0) residual_chunk_kernel<<<chunks, kThreads, 0, st>>>(d_obs, d_cal, d_res, n, scratch);
    sum_chunks_kernel<<<1, kThreads, 0, st>>>(scratch, chunks, scratch + kMaxPartials, d_sum);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        *err = std::string("fwi_residual_noalloc launch: ") + cudaGetErrorString(e);
        return -3;
    }
    return 0;
}

}  // namespace fwi
