// k_rbc.cu — random boundary velocity of every shot of a batch in one launch.
//
// Replaces random_boundary_bg + the per-point launches of random_boundary_gp
// (src/modeling/modeling.cu:431-531).  For each cell of a shot's padded grid:
//   1. outside the interior [nb, nzz-nb) x [nb, nxx-nb): the nearest interior
//      edge velocity plus f*varVp*N(0,1) per axis, f ramping from 1 at the outer
//      edge to 0 at the interior (random_boundary_bg);
//   2. outside the strict interior test X > nb*dh && X < x_max - nb*dh && ...
//      (so rows/columns nb and n-1-nb are included, as in the reference):
//      every Gaussian bump of the shot in sampling order, each followed by the
//      clamp to [vmin - varVp, vmax + varVp] (random_boundary_gp).
// The bumps are applied per cell in one loop instead of one full-grid launch
// per bump; each cell's sequence of operations is the reference's.
//
// This file is compiled with -fmad=false: with the counter-based normals and
// exp of detmath.h, every cell is bit-identical to a host evaluation.
#include <cuda_runtime.h>

#include "detmath.h"
#include "kernels.h"

namespace fwi {

namespace {

__global__ void rbc_kernel(RbcArgs a) {
    const int s = blockIdx.y;
    const int nxx = a.nxx[s];
    const long long cells = (long long)nxx * a.ldz;
    const float* base = a.base + (size_t)s * a.base_stride;
    float* out = a.out + (size_t)s * a.out_stride;
    const int b0 = a.bump_ptr[s], b1 = a.bump_ptr[s + 1];
    const uint32_t shot = (uint32_t)a.shot_id[s];
    const uint64_t kx = detm::stream_key(a.seed, shot, detm::STREAM_BG_X);
    const uint64_t kz = detm::stream_key(a.seed, shot, detm::STREAM_BG_Z);
    const int nb = a.nb, nzz = a.nzz;
    const float dh = a.dh;
    const float fnb = (float)(nb)*dh;
    const float x_max = (nxx - 1) * dh;
    const float z_max = (nzz - 1) * dh;
    const float vhi = a.vmax + a.varVp, vlo = a.vmin - a.varVp;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
         c += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(c / a.ldz), i = (int)(c - (long long)j * a.ldz);
        if (i >= nzz) { out[c] = 0.0f; continue; }
        float v = base[c];
        if (!((i >= nb) && (i < nzz - nb) && (j >= nb) && (j < nxx - nb))) {
            const int ii = min(max(i, nb), nzz - nb - 1);
            const int jj = min(max(j, nb), nxx - nb - 1);
            float val = base[(size_t)jj * a.ldz + ii];
            const uint64_t idx = (uint64_t)i + (uint64_t)j * (uint64_t)nzz;
            if (j < nb) {
                const float fx = 1.0f - (float)(j) / (float)(nb);
                val = val + fx * a.varVp * detm::normalf(kx, idx);
            } else if (j >= nxx - nb) {
                const float fx = 1.0f - (float)(nxx - j - 1) / (float)(nb);
                val = val + fx * a.varVp * detm::normalf(kx, idx);
            }
            if (i < nb) {
                const float fz = 1.0f - (float)(i) / (float)(nb);
                val = val + fz * a.varVp * detm::normalf(kz, idx);
            } else if (i >= nzz - nb) {
                const float fz = 1.0f - (float)(nzz - i - 1) / (float)(nb);
                val = val + fz * a.varVp * detm::normalf(kz, idx);
            }
            v = val;
        }
        const float X = (float)(j)*dh, Z = (float)(i)*dh;
        if (!((X > fnb) && (X < x_max - fnb) && (Z > fnb) && (Z < z_max - fnb))) {
            for (int p = b0; p < b1; ++p) {
                const BumpDev b = a.bumps[p];
                const float ax = (X - b.xc) / b.r, az = (Z - b.zc) / b.r;
                const float q = ax * ax + az * az;
                // exp(-0.5 q) rounds to 0.0f for q > 240: the addition is then a no-op
                if (q <= 240.0f) v = v + b.factor * b.A * detm::expf_nonpos(-0.5f * q);
                v = v > vhi ? vhi : v;
                v = v < vlo ? vlo : v;
            }
        }
        out[c] = v;
    }
}

}  // namespace

void launch_rbc(const RbcArgs& a, int nshots, cudaStream_t st) {
    const long long cells = (long long)a.max_nxx * a.ldz;
    int bx = (int)((cells + 255) / 256);
    if (bx > 4096) bx = 4096;
    rbc_kernel<<<dim3((unsigned)bx, (unsigned)nshots), 256, 0, st>>>(a);
}

}  // namespace fwi
