// Leapfrog updates on device-resident state (particle-id order, n x 3 FP64).
#include "common.cuh"
#include "kernels.h"

namespace fmmx {

// v += h * a
__global__ void k_kick(size_t n3, double* __restrict__ v, const double* __restrict__ a, double h) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x)
        v[i] += h * a[i];
}

// x += h * v
__global__ void k_drift(size_t n3, double* __restrict__ x, const double* __restrict__ v, double h) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x)
        x[i] += h * v[i];
}

// per-body time steps (n bodies, dt[b]): v += c * dt[b] * a  and  x += c * dt[b] * v
__global__ void k_kick_rows(size_t n3, double* __restrict__ v, const double* __restrict__ a,
                            const double* __restrict__ dt, double c) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x)
        v[i] += (c * dt[i / 3]) * a[i];
}
__global__ void k_drift_rows(size_t n3, double* __restrict__ x, const double* __restrict__ v,
                             const double* __restrict__ dt) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x)
        x[i] += dt[i / 3] * v[i];
}

}  // namespace fmmx
