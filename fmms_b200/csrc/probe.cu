// FMA-throughput probe: the roofline denominator of the CUDA-core kernels
// (FP64 for the plain form, FP32 for the mixed form). Eight independent FMA
// chains per thread, register resident, every SM fully occupied.
#include <cuda_runtime.h>

#include "../../include/fmmx.h"

namespace {
template <typename T>
__global__ void k_fma_loop(T* out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
            x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-1) out[0] = s;  // keeps the chains live
}

template <typename T>
double run(int nsm) {
    T* d = nullptr;
    cudaMalloc(&d, sizeof(T));
    const int threads = 256, blocks = nsm * 8, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_loop<T><<<blocks, threads>>>(d, 64, (T)0.999999, (T)1e-7);
    cudaEventRecord(e0);
    k_fma_loop<T><<<blocks, threads>>>(d, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    return flops / (ms * 1e-3) / 1e12;
}
}  // namespace

extern "C" fmmx_status fmmx_probe_fma_peak(int device, int fp64, double* tflops) {
    if (!tflops) return FMMX_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FMMX_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return FMMX_INVALID_ARG;
    cudaSetDevice(device);
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    *tflops = fp64 ? run<double>(nsm) : run<float>(nsm);
    return cudaGetLastError() == cudaSuccess ? FMMX_OK : FMMX_DEVICE_ERROR;
}
