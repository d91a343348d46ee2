// k_util.cu — grid padding / cropping, image and gradient post-processing,
// FP64 misfit reduction and model updates, all on the device so that a
// migration or an inversion iteration needs no host round trip.
#include <cuda_runtime.h>

#include "kernels.h"

namespace fwi {

namespace {

constexpr int kRedThreads = 256;

__global__ void expand_kernel(const float* __restrict__ model, int nz, int nx, float* __restrict__ out,
                              long long out_stride, const int* __restrict__ c0, const int* __restrict__ w, int nb,
                              int nzz, int ldz, int max_nxx) {
    const int s = blockIdx.y;
    const int ws = w[s], cs = c0[s];
    const int nxx = ws + 2 * nb;
    float* o = out + (size_t)s * out_stride;
    const long long cells = (long long)max_nxx * ldz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
         c += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(c / ldz), i = (int)(c - (long long)j * ldz);
        float v = 0.0f;
        if (i < nzz && j < nxx) {
            const int mi = min(max(i - nb, 0), nz - 1);
            const int mj = cs + min(max(j - nb, 0), ws - 1);
            v = model[(size_t)mj * nz + mi];
        }
        (void)nx;
        o[c] = v;
    }
}

__global__ void crop_sum_kernel(const float* __restrict__ padded, long long stride, int nshots, int nb, int ldz,
                                int nz, int nx, const int* __restrict__ c0, const int* __restrict__ w,
                                float* __restrict__ out, bool accumulate) {
    const long long n = (long long)nz * nx;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(c / nz), i = (int)(c - (long long)j * nz);
        float acc = accumulate ? out[c] : 0.0f;
        for (int s = 0; s < nshots; ++s) {
            const int lj = j - __ldg(c0 + s);
            if (lj < 0 || lj >= __ldg(w + s)) continue;
            acc += padded[(size_t)s * stride + (size_t)(lj + nb) * ldz + (i + nb)];
        }
        out[c] = acc;
    }
}

__global__ void mask_traces_kernel(float* __restrict__ data, const unsigned char* __restrict__ keep, size_t ntraces,
                                   int nt) {
    const size_t n = ntraces * (size_t)nt;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        if (!keep[c / nt]) data[c] = 0.0f;
}

__global__ void rtm_post_kernel(const float* __restrict__ img, const float* __restrict__ illum, int nz, int nx,
                                float idh2, float* __restrict__ out) {
    const long long n = (long long)nz * nx;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nz);
        float r = 0.0f;
        if (i > 0 && i < nz - 1) {
            const float qm = img[c - 1] / illum[c - 1];
            const float q0 = img[c] / illum[c];
            const float qp = img[c + 1] / illum[c + 1];
            r = -1.0f * (qm - 2.0f * q0 + qp) * idh2;
        }
        out[c] = r;
    }
}

__global__ void grad_post_kernel(const float* __restrict__ g, const float* __restrict__ illum, int nz, int nx,
                                 float idh2, int zmask_i, float* __restrict__ out, unsigned int* gmax_bits) {
    const long long n = (long long)nz * nx;
    float local = 0.0f;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nz);
        float r = 0.0f;
        if (i > zmask_i && i < nz - 1) {
            const float qm = g[c - 1] / illum[c - 1];
            const float q0 = g[c] / illum[c];
            const float qp = g[c + 1] / illum[c + 1];
            r = -1.0f * (qm - 2.0f * q0 + qp) * idh2;
        }
        out[c] = r;
        local = fmaxf(local, fabsf(r));
    }
    // max of non-negative floats == max of their bit patterns
    for (int o = 16; o > 0; o >>= 1) local = fmaxf(local, __shfl_xor_sync(0xffffffffu, local, o));
    if ((threadIdx.x & 31) == 0) atomicMax(gmax_bits, __float_as_uint(local));
}

__global__ void absmax_kernel(const float* __restrict__ x, size_t n, unsigned int* bits) {
    float m = 0.0f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(bits, __float_as_uint(m));
}

__global__ void scale_inv_kernel(float* x, size_t n, const unsigned int* gmax_bits) {
    const float inv = 1.0f / __uint_as_float(*gmax_bits);
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        x[c] *= inv;
}

__global__ void residual_kernel(const float* __restrict__ obs, const float* __restrict__ cal, float* __restrict__ res,
                                size_t n, double* __restrict__ partial) {
    __shared__ double red[kRedThreads / 32];
    double acc = 0.0;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const float r = obs[c] - cal[c];
        res[c] = r;
        acc += (double)r * (double)r;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kRedThreads / 32; ++w) t += red[w];
        partial[blockIdx.x] = t;
    }
}

__global__ void sum_partials_kernel(const double* __restrict__ partial, int n, double* out) {
    __shared__ double red[kRedThreads / 32];
    double acc = 0.0;
    for (int c = threadIdx.x; c < n; c += blockDim.x) acc += partial[c];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kRedThreads / 32; ++w) t += red[w];
        *out = t;
    }
}

__global__ void trial_kernel(const float* __restrict__ m, const float* __restrict__ g, float alpha,
                             float* __restrict__ vp, size_t n) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const float p = m[c] - alpha * g[c];
        vp[c] = 1.0f / sqrtf(p);
    }
}

__global__ void update_kernel(float* m, const float* __restrict__ g, float step, float* __restrict__ vp, size_t n,
                              float mlo, float mhi) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        float nm = m[c] - step * g[c];
        if (mlo > 0.0f) nm = fminf(fmaxf(nm, mlo), mhi);
        m[c] = nm;
        vp[c] = 1.0f / sqrtf(nm);
    }
}

__global__ void slowness2_kernel(const float* __restrict__ vp, float* __restrict__ m, size_t n) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        m[c] = 1.0f / (vp[c] * vp[c]);
}

__global__ void finite_kernel(const float* __restrict__ x, size_t n, int* flag) {
    bool bad = false;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        bad |= !isfinite(x[c]);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(flag, 1);
}

__global__ void inject_points_kernel(float* field, long long fstride, const ShotDesc* shots, InjTable inj,
                                     int ldz) {
    const int s = blockIdx.y;
    const ShotDesc sd = shots[s];
    float* f = field + (size_t)s * fstride;
    if (inj.sample < 0) return;
    // one thread per column: points of different columns never share a cell,
    // and a column's points are added in table order as in the step kernel
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < sd.nxx; j += gridDim.x * blockDim.x) {
        const int kb = inj.colptr[sd.col_off + j], ke = inj.colptr[sd.col_off + j + 1];
        for (int k = kb; k < ke; ++k)
            f[(size_t)j * ldz + inj.z[k]] += inj.scale * inj.series[inj.soff[k] + inj.sample];
    }
}

unsigned grid_for(size_t n, int threads = 256, unsigned cap = 148 * 16) {
    size_t b = (n + threads - 1) / threads;
    if (b == 0) b = 1;
    return (unsigned)(b < cap ? b : cap);
}

}  // namespace

void launch_expand(const float* model, int nz, int nx, float* out, long long out_stride, const int* c0,
                   const int* w, int nshots, int nb, int nzz, int ldz, int max_nxx, cudaStream_t st) {
    dim3 grid(grid_for((size_t)max_nxx * ldz), (unsigned)nshots);
    expand_kernel<<<grid, 256, 0, st>>>(model, nz, nx, out, out_stride, c0, w, nb, nzz, ldz, max_nxx);
}

void launch_crop_sum(const float* padded, long long stride, int nshots, int nb, int ldz, int nz, int nx,
                     const int* c0, const int* w, float* out, bool accumulate, cudaStream_t st) {
    crop_sum_kernel<<<grid_for((size_t)nz * nx), 256, 0, st>>>(padded, stride, nshots, nb, ldz, nz, nx, c0, w, out,
                                                               accumulate);
}

void launch_mask_traces(float* data, const unsigned char* keep, size_t ntraces, int nt, cudaStream_t st) {
    mask_traces_kernel<<<grid_for(ntraces * (size_t)nt), 256, 0, st>>>(data, keep, ntraces, nt);
}

void launch_rtm_post(const float* img, const float* illum, int nz, int nx, float idh2, float* out,
                     cudaStream_t st) {
    rtm_post_kernel<<<grid_for((size_t)nz * nx), 256, 0, st>>>(img, illum, nz, nx, idh2, out);
}

void launch_grad_post(const float* g, const float* illum, int nz, int nx, float idh2, int zmask_i, float* out,
                      unsigned int* gmax_bits, cudaStream_t st) {
    cudaMemsetAsync(gmax_bits, 0, sizeof(unsigned int), st);
    grad_post_kernel<<<grid_for((size_t)nz * nx), 256, 0, st>>>(g, illum, nz, nx, idh2, zmask_i, out, gmax_bits);
}

void launch_absmax(const float* x, size_t n, unsigned int* bits, cudaStream_t st) {
    cudaMemsetAsync(bits, 0, sizeof(unsigned int), st);
    absmax_kernel<<<grid_for(n), 256, 0, st>>>(x, n, bits);
}

void launch_scale_by_inverse(float* x, size_t n, const unsigned int* gmax_bits, cudaStream_t st) {
    scale_inv_kernel<<<grid_for(n), 256, 0, st>>>(x, n, gmax_bits);
}

int residual_blocks(size_t n) { return (int)grid_for(n, kRedThreads, 148 * 8); }

void launch_residual(const float* obs, const float* cal, float* res, size_t n, double* partial, double* out,
                     cudaStream_t st) {
    const int nb = residual_blocks(n);
    residual_kernel<<<nb, kRedThreads, 0, st>>>(obs, cal, res, n, partial);
    sum_partials_kernel<<<1, kRedThreads, 0, st>>>(partial, nb, out);
}

void launch_trial_velocity(const float* m, const float* g, float alpha, float* vp, size_t n, cudaStream_t st) {
    trial_kernel<<<grid_for(n), 256, 0, st>>>(m, g, alpha, vp, n);
}

void launch_update_model(float* m, const float* g, float step, float* vp, size_t n, cudaStream_t st, float mlo,
                         float mhi) {
    update_kernel<<<grid_for(n), 256, 0, st>>>(m, g, step, vp, n, mlo, mhi);
}

void launch_slowness2(const float* vp, float* m, size_t n, cudaStream_t st) {
    slowness2_kernel<<<grid_for(n), 256, 0, st>>>(vp, m, n);
}

void launch_check_finite(const float* x, size_t n, int* flag, cudaStream_t st) {
    finite_kernel<<<grid_for(n), 256, 0, st>>>(x, n, flag);
}

void launch_inject_points(float* field, long long fstride, const ShotDesc* shots, int nshots, InjTable inj,
                          int ldz, cudaStream_t st) {
    inject_points_kernel<<<dim3(8, nshots), 256, 0, st>>>(field, fstride, shots, inj, ldz);
}

}  // namespace fwi
