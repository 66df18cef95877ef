// Directed, destination-segmented interaction lists.
//
// The walk emits mutual pairs, as the reference's recorder does
// (walk.rs:342-488). The evaluation kernels here are destination-owned (one
// CTA or warp writes each cell's locals or each leaf's bodies, no atomics), so
// every mutual pair (a, b) becomes the two directed entries a->b and b->a, a
// leaf self pair one entry. The lists are built by a counting sort on the
// destination -- count the entries per destination, scan the counts into
// segment offsets, scatter every source into its destination's segment --
// followed by a sort of each segment's sources (a bitonic network per
// segment, in shared memory). The entries of destination c
// are then its sources in ascending order, src[off[c] .. off[c+1]), whatever
// order the walk's atomics appended the pairs in, which fixes the
// accumulation order and so every result bit.
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "kernels.h"

namespace fmmx {

// entries per destination; P2P self pairs count once and every pair adds its
// directed body-body interactions (|A|(|A|-1) for a self pair, 2|A||B| else)
__global__ void k_count_dst(const uint2* __restrict__ pairs, int np, uint32_t* __restrict__ cnt,
                            const uint32_t* __restrict__ body_count, unsigned long long* __restrict__ interactions) {
    unsigned long long local = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
        const uint2 pr = pairs[q];
        atomicAdd(&cnt[pr.y], 1u);
        if (pr.x != pr.y) atomicAdd(&cnt[pr.x], 1u);
        if (body_count) {
            const unsigned long long ca = body_count[pr.x], cb = body_count[pr.y];
            local += pr.x == pr.y ? ca * (ca - 1) : 2ull * ca * cb;
        }
    }
    if (body_count) {
        for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
        if ((threadIdx.x & 31) == 0 && local) atomicAdd(interactions, local);
    }
}

// every source into its destination's segment (slots taken by counting the
// destination's remaining count down; the order within a segment is fixed
// afterwards by the segment sort)
__global__ void k_scatter_dst(const uint2* __restrict__ pairs, int np, const uint32_t* __restrict__ off,
                              uint32_t* __restrict__ left, uint32_t* __restrict__ src) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
        const uint2 pr = pairs[q];
        src[off[pr.y] + atomicSub(&left[pr.y], 1u) - 1u] = pr.x;  // a -> b
        if (pr.x != pr.y) src[off[pr.x] + atomicSub(&left[pr.x], 1u) - 1u] = pr.y;  // b -> a
    }
}

// Ascending sort of a[0..n) by a bitonic network over P = 2^k >= n slots in
// which every comparator puts the smaller value at the lower index (the first
// step of each merge compares mirrored positions, the others i with i + h).
// Slots n..P-1 act as +infinity: a comparator whose upper slot is one of them
// never swaps, so they are never read or written. All threads of the block
// call it; `a` is shared or global memory of this block only.
__device__ void bitonic_sort_block(uint32_t* a, int n) {
    int P = 1;
    while (P < n) P <<= 1;
    for (int size = 2; size <= P; size <<= 1) {
        const int hs = size >> 1;
        for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
            const int i = (t / hs) * size + (t % hs);
            const int j = (t / hs) * size + size - 1 - (t % hs);
            if (j < n) {
                const uint32_t x = a[i], y = a[j];
                if (x > y) {
                    a[i] = y;
                    a[j] = x;
                }
            }
        }
        __syncthreads();
        for (int h = hs >> 1; h > 0; h >>= 1) {
            for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
                const int i = (t / h) * 2 * h + (t % h);
                const int j = i + h;
                if (j < n) {
                    const uint32_t x = a[i], y = a[j];
                    if (x > y) {
                        a[i] = y;
                        a[j] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

#define SEG_SMALL 2048
#define SEG_LARGE_SMEM 32768

// One block per destination: segments of up to SEG_SMALL entries are sorted in
// shared memory into `out`; longer ones are appended to `big` for
// k_sort_segments_large.
__global__ void __launch_bounds__(256) k_sort_segments(const uint32_t* __restrict__ off, int nseg,
                                                       const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                       int* __restrict__ big, int* __restrict__ nbig) {
    __shared__ uint32_t buf[SEG_SMALL];
    const int c = blockIdx.x;
    if (c >= nseg) return;
    const uint32_t b = off[c];
    const int n = (int)(off[c + 1] - b);
    if (n == 0) return;
    if (n > SEG_SMALL) {
        if (threadIdx.x == 0) big[atomicAdd(nbig, 1)] = c;
        return;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) buf[i] = in[b + i];
    __syncthreads();
    if (n > 1) bitonic_sort_block(buf, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) out[b + i] = buf[i];
}

// The longer segments (a few fat leaves with thousands of neighbours): in
// shared memory up to SEG_LARGE_SMEM entries, in place in `out` beyond.
__global__ void __launch_bounds__(1024) k_sort_segments_large(const uint32_t* __restrict__ off,
                                                              const uint32_t* __restrict__ in,
                                                              uint32_t* __restrict__ out, const int* __restrict__ big,
                                                              const int* __restrict__ nbig) {
    extern __shared__ uint32_t sbuf[];
    const int nb = *nbig;
    for (int q = blockIdx.x; q < nb; q += gridDim.x) {
        const int c = big[q];
        const uint32_t b = off[c];
        const int n = (int)(off[c + 1] - b);
        uint32_t* a = n <= SEG_LARGE_SMEM ? sbuf : out + b;
        for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = in[b + i];
        __syncthreads();
        bitonic_sort_block(a, n);
        if (n <= SEG_LARGE_SMEM)
            for (int i = threadIdx.x; i < n; i += blockDim.x) out[b + i] = a[i];
        __syncthreads();
    }
}

cudaError_t scan_u32(void* tmp, size_t tmp_bytes, const uint32_t* in, uint32_t* out, int n, cudaStream_t s) {
    return cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, n, s);
}

size_t directed_list_temp(int nitems, int ncells) {
    (void)nitems;
    size_t a = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, a, (const uint32_t*)nullptr, (uint32_t*)nullptr, ncells + 1);
    // after the scan's storage: the count and the ids of the long segments
    return ((a + 255) / 256) * 256 + sizeof(int) * ((size_t)ncells + 64);
}

cudaError_t build_directed_list(void* tmp, size_t tmp_bytes, const uint2* pairs, int np, int nitems, int ncells,
                                const uint32_t* body_count, unsigned long long* interactions, uint32_t* cnt,
                                uint32_t* off, uint32_t* src_unsorted, uint32_t* src, unsigned grid,
                                cudaStream_t s) {
    (void)nitems;
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt, off, ncells + 1, s);
    const size_t big_at = ((scan_bytes + 255) / 256) * 256;
    if (tmp_bytes < big_at + sizeof(int) * ((size_t)ncells + 64)) return cudaErrorInvalidValue;
    int* nbig = reinterpret_cast<int*>(static_cast<char*>(tmp) + big_at);
    int* big = nbig + 64;
    cudaError_t e = cudaMemsetAsync(cnt, 0, (size_t)(ncells + 1) * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (np > 0) k_count_dst<<<grid, 256, 0, s>>>(pairs, np, cnt, body_count, interactions);
    e = cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, cnt, off, ncells + 1, s);
    if (e != cudaSuccess || np == 0) return e;
    k_scatter_dst<<<grid, 256, 0, s>>>(pairs, np, off, cnt, src_unsorted);
    e = cudaMemsetAsync(nbig, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    k_sort_segments<<<ncells, 256, 0, s>>>(off, ncells, src_unsorted, src, big, nbig);
    e = cudaFuncSetAttribute(k_sort_segments_large, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             SEG_LARGE_SMEM * (int)sizeof(uint32_t));  // 128 KB, on the current device
    if (e != cudaSuccess) return e;
    k_sort_segments_large<<<148, 1024, SEG_LARGE_SMEM * sizeof(uint32_t), s>>>(off, src_unsorted, src, big, nbig);
    return cudaGetLastError();
}

}  // namespace fmmx
