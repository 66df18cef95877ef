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

}  // namespace fmmx
