// k_prep.cu — GPU data preparation that the reference does in Python before
// RTM and FWI, moved next to the data:
//
//   * direct-wave mute (run/generate_input_data.py:22-44): every shot is
//     normalised by its largest |amplitude|, then the samples t < tId[r] of
//     trace r are tapered by exp(-0.5 ((t - tId[r]) / gstd)^2), with
//     tId[r] = int((distance_r / velocity + delay) / dt);
//   * initial model (run/generate_setup.py:49-51): vp_init = 1 / G(1 / vp),
//     G = scipy.ndimage.gaussian_filter (separable, mode 'reflect', radius
//     int(4 sigma + 0.5)), first along z then along x with a float32
//     intermediate; the rows above depth_mask keep vp.
//
// Arithmetic follows the scripts' numpy dtypes: the normalisation and tId in
// float32 (explicitly rounded operations, no contraction), the taper and the
// filter sums in float64 rounded once to float32.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace fwi {

namespace {

unsigned grid_of(size_t n, int threads = 256, unsigned cap = 148 * 16) {
    size_t b = (n + threads - 1) / threads;
    if (b == 0) b = 1;
    return (unsigned)(b < cap ? b : cap);
}

// max |x| of every shot's block (nonnegative floats order like their bits)
__global__ void shot_absmax_kernel(const float* __restrict__ data, size_t per_shot, unsigned* __restrict__ bits) {
    const int s = blockIdx.y;
    const float* d = data + (size_t)s * per_shot;
    float m = 0.0f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < per_shot; i += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(d[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(bits + s, __float_as_uint(m));
}

// trace r of shot s: normalise, then taper samples t < tid
__global__ void mute_kernel(float* __restrict__ data, int nt, int nrec, const unsigned* __restrict__ bits,
                            const float* __restrict__ sx, const float* __restrict__ sz, const float* __restrict__ rx,
                            const float* __restrict__ rz, float velocity, float delay, float dt, double gstd) {
    const int s = blockIdx.y;
    const float inv = __fdiv_rn(1.0f, __uint_as_float(bits[s]));
    for (int r = blockIdx.x; r < nrec; r += gridDim.x) {
        const float dx = __fsub_rn(rx[r], sx[s]);
        const float dz = __fsub_rn(rz[r], sz[s]);
        const float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)));
        const float tf = __fdiv_rn(__fadd_rn(__fdiv_rn(dist, velocity), delay), dt);
        const long long tid = (long long)tf;  // truncation, as numpy's astype(int)
        float* tr = data + ((size_t)s * nrec + r) * nt;
        for (int t = threadIdx.x; t < nt; t += blockDim.x) {
            float v = __fmul_rn(tr[t], inv);
            if (t < tid) {
                const double q = (double)(t - tid) / gstd;
                const double w = exp(__dmul_rn(-0.5, __dmul_rn(q, q)));
                v = (float)__dmul_rn((double)v, w);
            }
            tr[t] = v;
        }
    }
}

__device__ __forceinline__ int reflect(int i, int n) {
    // scipy.ndimage 'reflect' (d c b a | a b c d | d c b a), any distance
    const int p = 2 * n;
    i %= p;
    if (i < 0) i += p;
    return i < n ? i : p - 1 - i;
}

// One gaussian_filter1d pass of an nz x nx (z fastest) array along z
// (axis 0) or x (axis 1); in is float32, the sum double, out float32.
// Symmetric kernels sum as scipy's correlate1d: centre first, then the pairs
// from the outermost inwards.
template <bool ALONG_Z>
__global__ void gauss_pass_kernel(const float* __restrict__ in, float* __restrict__ out, int nz, int nx,
                                  const double* __restrict__ w, int radius, bool recip_in) {
    const size_t n = (size_t)nz * nx;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(c / nz), i = (int)(c - (size_t)j * nz);
        auto at = [&](int k) -> double {
            const float x = ALONG_Z ? in[(size_t)j * nz + reflect(i + k, nz)] : in[(size_t)reflect(j + k, nx) * nz + i];
            return (double)(recip_in ? __fdiv_rn(1.0f, x) : x);
        };
        double acc = __dmul_rn(at(0), w[0]);
        for (int k = radius; k >= 1; --k) acc = __dadd_rn(acc, __dmul_rn(__dadd_rn(at(-k), at(k)), w[k]));
        out[c] = (float)acc;
    }
}

// vp_init = 1 / smoothed below row keep_rows, vp above
__global__ void recip_keep_kernel(const float* __restrict__ smooth, const float* __restrict__ vp, int nz, int nx,
                                  int keep_rows, float* __restrict__ out) {
    const size_t n = (size_t)nz * nx;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nz);
        out[c] = i < keep_rows ? vp[c] : __fdiv_rn(1.0f, smooth[c]);
    }
}

}  // namespace

void launch_mute_direct(float* data, int nsrc, int nrec, int nt, const float* sx, const float* sz, const float* rx,
                        const float* rz, float velocity, float delay, float dt, float gstd, unsigned* bits,
                        cudaStream_t st) {
    const size_t per = (size_t)nrec * nt;
    cudaMemsetAsync(bits, 0, nsrc * sizeof(unsigned), st);
    shot_absmax_kernel<<<dim3(grid_of(per, 256, 64), nsrc), 256, 0, st>>>(data, per, bits);
    mute_kernel<<<dim3(nrec < 1024 ? nrec : 1024, nsrc), 256, 0, st>>>(data, nt, nrec, bits, sx, sz, rx, rz, velocity,
                                                                      delay, dt, (double)gstd);
}

void launch_smooth_slowness(const float* vp, int nz, int nx, const double* weights, int radius, int keep_rows,
                            float* tmp, float* out, cudaStream_t st) {
    const size_t n = (size_t)nz * nx;
    gauss_pass_kernel<true><<<grid_of(n), 256, 0, st>>>(vp, out, nz, nx, weights, radius, true);
    gauss_pass_kernel<false><<<grid_of(n), 256, 0, st>>>(out, tmp, nz, nx, weights, radius, false);
    recip_keep_kernel<<<grid_of(n), 256, 0, st>>>(tmp, vp, nz, nx, keep_rows, out);
}

}  // namespace fwi
