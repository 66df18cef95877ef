// FP64 direct sum at selected target bodies: the error harness's exact
// reference (direct.rs:6-31 one-sided, and the sampled error of
// crates/bench/src/main.rs:34-78). Sources are split across blockIdx.y; each
// split writes its partial sums and k_direct_reduce adds them in split order,
// so the result is deterministic.
#include "common.cuh"
#include "kernels.h"

namespace fmmx {

#define DIR_BLOCK 128

__global__ void __launch_bounds__(DIR_BLOCK) k_direct_targets(const double* __restrict__ pos,
                                                              const double* __restrict__ mass, size_t n,
                                                              const uint32_t* __restrict__ tgt, size_t nt,
                                                              double soft2, double* __restrict__ part) {
    __shared__ double sx[DIR_BLOCK], sy[DIR_BLOCK], sz[DIR_BLOCK], sm[DIR_BLOCK];
    const size_t q = blockIdx.x * (size_t)DIR_BLOCK + threadIdx.x;
    const bool active = q < nt;
    const uint32_t ti = active ? tgt[q] : 0;
    const double xi = active ? pos[3 * (size_t)ti] : 0.0;
    const double yi = active ? pos[3 * (size_t)ti + 1] : 0.0;
    const double zi = active ? pos[3 * (size_t)ti + 2] : 0.0;
    const size_t per = (n + gridDim.y - 1) / gridDim.y;
    const size_t j0 = blockIdx.y * per, j1 = min(n, j0 + per);
    double ax = 0, ay = 0, az = 0, ph = 0, f = 0;
    for (size_t b0 = j0; b0 < j1; b0 += DIR_BLOCK) {
        const size_t j = b0 + threadIdx.x;
        if (j < j1) {
            sx[threadIdx.x] = pos[3 * j];
            sy[threadIdx.x] = pos[3 * j + 1];
            sz[threadIdx.x] = pos[3 * j + 2];
            sm[threadIdx.x] = mass[j];
        }
        __syncthreads();
        const int nb = (int)min((size_t)DIR_BLOCK, j1 - b0);
        if (active) {
            for (int k = 0; k < nb; ++k) {
                if (b0 + k == ti) continue;
                const double dx = sx[k] - xi, dy = sy[k] - yi, dz = sz[k] - zi;
                const double r2 = dx * dx + dy * dy + dz * dz + soft2;
                const double inv = 1.0 / sqrt(r2);
                const double inv2 = inv * inv;
                const double inv3 = inv2 * inv;
                ax += sm[k] * inv3 * dx;
                ay += sm[k] * inv3 * dy;
                az += sm[k] * inv3 * dz;
                f += sm[k] * inv2;
                ph += sm[k] * inv;
            }
        }
        __syncthreads();
    }
    if (active) {
        double* o = part + ((size_t)blockIdx.y * nt + q) * 5;
        o[0] = ax;
        o[1] = ay;
        o[2] = az;
        o[3] = ph;
        o[4] = f;
    }
}

__global__ void k_direct_reduce(const double* __restrict__ part, int nsplit, size_t nt, double* __restrict__ acc,
                                double* __restrict__ pot, double* __restrict__ fsc) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nt; q += (size_t)gridDim.x * blockDim.x) {
        double s[5] = {0, 0, 0, 0, 0};
        for (int b = 0; b < nsplit; ++b)
            for (int k = 0; k < 5; ++k) s[k] += part[((size_t)b * nt + q) * 5 + k];
        acc[3 * q] = s[0];
        acc[3 * q + 1] = s[1];
        acc[3 * q + 2] = s[2];
        if (pot) pot[q] = s[3];
        if (fsc) fsc[q] = s[4];
    }
}

}  // namespace fmmx
