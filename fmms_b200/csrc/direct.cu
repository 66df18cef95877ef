// FP64 direct sum at selected target bodies: the error harness's exact
// reference (direct.rs:6-31 one-sided, and the sampled error of
// crates/bench/src/main.rs:34-78). Sources are split across blockIdx.y; each
// split writes its partial sums and k_direct_reduce adds them in split order,
// so the result is deterministic.
#include <mutex>

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

// ---------------------------------------------------------------------------
// Allocation-free direct sum (no counterpart in the reference).
//
// For callers that cannot allocate device memory: a physics step running in a
// fixed-latency frame loop (cudaMalloc and cudaFree can block and synchronise
// the whole device, so a per-frame allocation shows up as a frame hitch), and
// hosts whose device memory is handed out by their own pool allocator, which
// owns the budget and forbids other allocations. Inputs and outputs are the
// caller's device buffers; the only other memory, the per-split partial sums,
// is the file-scope array below, sized for FMMX_DIRECT_NOALLOC_MAX_TARGETS
// targets and held by every GPU that loads this library until the process
// exits.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address (cudaGetSymbolAddress) and caches it; make that first
// call before any stream capture. Calls share the array and each call writes
// every partial it reads, so nothing needs clearing between calls; calls that
// overlap on the GPU (different streams, no ordering) race on it.
#define FMMX_NOALLOC_NSPLIT 32
#define FMMX_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double
    g_direct_scratch[(size_t)FMMX_DIRECT_NOALLOC_MAX_TARGETS * FMMX_NOALLOC_NSPLIT * 5];

namespace {
std::mutex g_scratch_mu;
double* g_scratch_addr[FMMX_NOALLOC_MAX_DEVICES] = {nullptr};
}  // namespace

namespace fmmx {

// k_direct_targets with a bound check on the target ids, which live in device
// memory here and cannot be validated on the host: an id >= n gives NaN.
__global__ void __launch_bounds__(DIR_BLOCK) k_direct_targets_checked(const double* __restrict__ pos,
                                                                      const double* __restrict__ mass, size_t n,
                                                                      const uint32_t* __restrict__ tgt, size_t nt,
                                                                      double soft2, double* __restrict__ part) {
    __shared__ double sx[DIR_BLOCK], sy[DIR_BLOCK], sz[DIR_BLOCK], sm[DIR_BLOCK];
    const size_t q = blockIdx.x * (size_t)DIR_BLOCK + threadIdx.x;
    const bool in_range = q < nt;
    const uint32_t t_raw = in_range ? tgt[q] : 0;
    const bool valid = in_range && (size_t)t_raw < n;
    const uint32_t ti = valid ? t_raw : 0;
    const double xi = valid ? pos[3 * (size_t)ti] : 0.0;
    const double yi = valid ? pos[3 * (size_t)ti + 1] : 0.0;
    const double zi = valid ? pos[3 * (size_t)ti + 2] : 0.0;
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
        if (valid) {
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
    if (in_range) {
        double* o = part + ((size_t)blockIdx.y * nt + q) * 5;
        const double bad = valid ? 0.0 : NAN;
        o[0] = ax + bad;
        o[1] = ay + bad;
        o[2] = az + bad;
        o[3] = ph + bad;
        o[4] = f + bad;
    }
}

}  // namespace fmmx

extern "C" fmmx_status fmmx_direct_targets_noalloc(int device, void* stream, size_t n, const double* d_pos,
                                                   const double* d_mass, double softening, size_t nt,
                                                   const uint32_t* d_targets, double* d_acc, double* d_pot,
                                                   double* d_fscale) {
    if (!d_pos || !d_mass || !d_targets || !d_acc || n == 0) return FMMX_INVALID_ARG;
    if (nt > FMMX_DIRECT_NOALLOC_MAX_TARGETS) return FMMX_INVALID_ARG;  // beyond the static scratch
    if (nt == 0) return FMMX_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FMMX_NO_DEVICE;
    }
    if (device < 0 || device >= ndev || device >= FMMX_NOALLOC_MAX_DEVICES) return FMMX_INVALID_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return FMMX_DEVICE_ERROR;
    }
    fmmx_status st = FMMX_OK;
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_addr[device]) {
            void* addr = nullptr;
            if (cudaGetSymbolAddress(&addr, g_direct_scratch) != cudaSuccess || addr == nullptr) {
                cudaGetLastError();
                st = FMMX_DEVICE_ERROR;
            } else {
                g_scratch_addr[device] = static_cast<double*>(addr);
            }
        }
        scratch = g_scratch_addr[device];
    }
    // an error left by earlier, unrelated work on this thread is not this
    // call's: report it without launching and leave it for its owner (peek,
    // do not clear); after that, an error is one of the launches below
    if (st == FMMX_OK && cudaPeekAtLastError() != cudaSuccess) st = FMMX_DEVICE_ERROR;
    if (st == FMMX_OK) {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        dim3 g((unsigned)((nt + DIR_BLOCK - 1) / DIR_BLOCK), FMMX_NOALLOC_NSPLIT);
        fmmx::k_direct_targets_checked<<<g, DIR_BLOCK, 0, s>>>(d_pos, d_mass, n, d_targets, nt,
                                                               softening * softening, scratch);
        if (cudaGetLastError() != cudaSuccess) st = FMMX_DEVICE_ERROR;
        if (st == FMMX_OK) {
            fmmx::k_direct_reduce<<<fmmx::grid_for(nt, 128), 128, 0, s>>>(scratch, FMMX_NOALLOC_NSPLIT, nt, d_acc,
                                                                          d_pot, d_fscale);
            if (cudaGetLastError() != cudaSuccess) st = FMMX_DEVICE_ERROR;
        }
    }
    cudaSetDevice(prev);
    return st;
}
