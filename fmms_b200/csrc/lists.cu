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
// segment, in registers). The entries of destination c
// are then its sources in ascending order, src[off[c] .. off[c+1]), whatever
// order the walk's atomics appended the pairs in, which fixes the
// accumulation order and so every result bit.
#include <atomic>

#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_radix_sort.cuh>

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

// ---------------------------------------------------------------- segment sort
// Ascending sorts by a bitonic network in which every comparator puts the
// smaller value at the lower index: merge stage `size` starts with a mirror
// step (e against e ^ (size - 1)) and continues with half-cleaners (e
// against e ^ h, h = size/4 .. 1). A warp holds a chunk of 32 R elements,
// element e = lane * R + j in register v[j]: steps with h < R are register
// compares, the others shuffles between lanes. Slots past the segment hold
// 0xffffffff (never a cell id), so they sort to the end.
__device__ __forceinline__ void cmp_up(uint32_t& lo, uint32_t& hi) {
    const uint32_t a = min(lo, hi), b = max(lo, hi);
    lo = a;
    hi = b;
}

// Every step distance is a template argument, so the register array is
// indexed by constants only (no local-memory copy of it).
// half-cleaner at distance H within the warp's chunk
template <int R, int H>
__device__ __forceinline__ void warp_half(uint32_t (&v)[R], int lane) {
    if constexpr (H < R) {
#pragma unroll
        for (int j = 0; j < R; ++j)
            if ((j & H) == 0) cmp_up(v[j], v[j | H]);
    } else {
        constexpr int lm = H / R;
        const bool low = (lane & lm) == 0;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const uint32_t o = __shfl_xor_sync(0xffffffffu, v[j], lm);
            v[j] = low ? min(v[j], o) : max(v[j], o);
        }
    }
}

// half-cleaners H, H/2, .., 1
template <int R, int H>
__device__ __forceinline__ void warp_clean(uint32_t (&v)[R], int lane) {
    warp_half<R, H>(v, lane);
    if constexpr (H > 1) warp_clean<R, H / 2>(v, lane);
}

// mirror step of merge stage SIZE (SIZE <= 32 R)
template <int R, int SIZE>
__device__ __forceinline__ void warp_mirror(uint32_t (&v)[R], int lane) {
    if constexpr (SIZE <= R) {
#pragma unroll
        for (int j = 0; j < R; ++j)
            if (j < (j ^ (SIZE - 1))) cmp_up(v[j], v[j ^ (SIZE - 1)]);
    } else {
        constexpr int lm = SIZE / R - 1;
        const bool low = (lane & (SIZE / R / 2)) == 0;
        uint32_t o[R];
#pragma unroll
        for (int j = 0; j < R; ++j) o[j] = __shfl_xor_sync(0xffffffffu, v[R - 1 - j], lm);
#pragma unroll
        for (int j = 0; j < R; ++j) v[j] = low ? min(v[j], o[j]) : max(v[j], o[j]);
    }
}

// merge stages SIZE .. 32 R: the full sort of the warp's 32 R elements from SIZE = 2
template <int R, int SIZE = 2>
__device__ __forceinline__ void warp_sort(uint32_t (&v)[R], int lane) {
    warp_mirror<R, SIZE>(v, lane);
    if constexpr (SIZE >= 4) warp_clean<R, SIZE / 4>(v, lane);
    if constexpr (SIZE < 32 * R) warp_sort<R, 2 * SIZE>(v, lane);
}

// the half-cleaners h = 512 .. 1 of a merge stage, on a 1024-element chunk
__device__ __forceinline__ void warp_clean_1024(uint32_t (&v)[32], int lane) { warp_clean<32, 512>(v, lane); }

template <int R>
__device__ __forceinline__ void warp_sort_segment(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int n,
                                                  int lane) {
    uint32_t v[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const int e = lane * R + j;
        v[j] = e < n ? in[e] : 0xffffffffu;
    }
    warp_sort<R>(v, lane);
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const int e = lane * R + j;
        if (e < n) out[e] = v[j];
    }
}

#define SEG_WARP 1024
#define SEG_MID 4096  // 1024 < n <= SEG_MID: blocks of 4 warps, the segment in 16 KB of shared memory;
                      // longer: CUB's segmented radix sort, one block per segment (sort_long_segments)

// One warp per destination: segments of up to SEG_WARP entries are sorted in
// registers into `out`; longer ones are appended to `mid` (up to SEG_MID) or
// `big` for the block kernels.
__global__ void __launch_bounds__(256) k_sort_segments(const uint32_t* __restrict__ off, int nseg,
                                                       const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                       int* __restrict__ mid, int* __restrict__ nmid,
                                                       int* __restrict__ big, int* __restrict__ nbig) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nseg; c += warps) {
        const uint32_t b = off[c];
        const int n = (int)(off[c + 1] - b);
        if (n == 0) continue;
        if (n > SEG_WARP) {
            if (lane == 0) {
                if (n <= SEG_MID) mid[atomicAdd(nmid, 1)] = c;
                else big[atomicAdd(nbig, 1)] = c;
            }
            continue;
        }
        const uint32_t* src = in + b;
        uint32_t* dst = out + b;
        if (n <= 32) warp_sort_segment<1>(src, dst, n, lane);
        else if (n <= 64) warp_sort_segment<2>(src, dst, n, lane);
        else if (n <= 128) warp_sort_segment<4>(src, dst, n, lane);
        else if (n <= 256) warp_sort_segment<8>(src, dst, n, lane);
        else if (n <= 512) warp_sort_segment<16>(src, dst, n, lane);
        else warp_sort_segment<32>(src, dst, n, lane);
    }
}

// The longer segments (leaves in dense cluster cores with thousands of
// neighbours), one block each: every warp sorts 1024-element chunks in
// registers; the merge stages above 1024 run their steps across chunks
// (distance >= 1024) on the whole segment, block-synchronised, and the steps
// within chunks again in registers. The segment is in shared memory up to
// SMEM_ENTRIES entries, in place in `out` beyond; slots from n up to the
// power of two are virtual (+infinity: never read or written).
template <int THREADS, int SMEM_ENTRIES>
__global__ void __launch_bounds__(THREADS) k_sort_segments_large(const uint32_t* __restrict__ off,
                                                                 const uint32_t* __restrict__ in,
                                                                 uint32_t* __restrict__ out,
                                                                 const int* __restrict__ big,
                                                                 const int* __restrict__ nbig) {
    extern __shared__ uint32_t sbuf[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = THREADS >> 5;
    const int nb = *nbig;
    for (int q = blockIdx.x; q < nb; q += gridDim.x) {
        const int c = big[q];
        const uint32_t b = off[c];
        const int n = (int)(off[c + 1] - b);
        uint32_t* a = n <= SMEM_ENTRIES ? sbuf : out + b;
        int P = SEG_WARP;
        while (P < n) P <<= 1;
        const int nchunk = P / SEG_WARP;
        // chunks sorted in registers
        for (int ch = wid; ch < nchunk; ch += nw) {
            uint32_t v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int e = ch * SEG_WARP + lane * 32 + j;
                v[j] = e < n ? in[b + e] : 0xffffffffu;
            }
            warp_sort<32>(v, lane);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int e = ch * SEG_WARP + lane * 32 + j;
                if (e < n) a[e] = v[j];
            }
        }
        __syncthreads();
        for (int size = 2 * SEG_WARP; size <= P; size <<= 1) {
            // steps across chunks: the mirror step, then half-cleaners h >= 1024
            for (int h = size / 2; h >= SEG_WARP; h >>= 1) {
                const bool mirror = h == size / 2;
                for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
                    int i, j;
                    if (mirror) {
                        i = (t / h) * size + (t % h);
                        j = (t / h) * size + size - 1 - (t % h);
                    } else {
                        i = (t / h) * 2 * h + (t % h);
                        j = i + h;
                    }
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
            // the remaining half-cleaners stay within chunks
            for (int ch = wid; ch < nchunk; ch += nw) {
                uint32_t v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int e = ch * SEG_WARP + lane * 32 + j;
                    v[j] = e < n ? a[e] : 0xffffffffu;
                }
                warp_clean_1024(v, lane);
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int e = ch * SEG_WARP + lane * 32 + j;
                    if (e < n) a[e] = v[j];
                }
            }
            __syncthreads();
        }
        if (n <= SMEM_ENTRIES)
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
    return a;
}

cudaError_t build_directed_list(void* tmp, size_t tmp_bytes, const uint2* pairs, int np, int nitems, int ncells,
                                const uint32_t* body_count, unsigned long long* interactions, uint32_t* cnt,
                                uint32_t* off, uint32_t* src_unsorted, uint32_t* src, int* longs, unsigned grid,
                                cudaStream_t s) {
    (void)nitems;
    int* nbig = longs;  // [0] long segments, [32] middle ones
    int* nmid = longs + 32;
    int* big = longs + 128;
    int* mid = big + ncells;
    cudaError_t e = cudaMemsetAsync(longs, 0, 128 * sizeof(int), s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(cnt, 0, (size_t)(ncells + 1) * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (np > 0) k_count_dst<<<grid, 256, 0, s>>>(pairs, np, cnt, body_count, interactions);
    size_t bytes = tmp_bytes;
    e = cub::DeviceScan::ExclusiveSum(tmp, bytes, cnt, off, ncells + 1, s);
    if (e != cudaSuccess || np == 0) return e;
    k_scatter_dst<<<grid, 256, 0, s>>>(pairs, np, off, cnt, src_unsorted);
    k_sort_segments<<<grid_for((size_t)ncells * 32, 256, 64u * g_nsm), 256, 0, s>>>(off, ncells, src_unsorted, src,
                                                                                   mid, nmid, big, nbig);
    // exactly the resident blocks, so the middle segments are spread over
    // blocks that all run at once
    static std::atomic<int> large_per_sm{0};
    if (large_per_sm.load() == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sort_segments_large<128, SEG_MID>, 128,
                                                          SEG_MID * sizeof(uint32_t)) != cudaSuccess ||
            b < 1)
            b = 1;
        large_per_sm.store(b);
    }
    const unsigned large_grid = (unsigned)(large_per_sm.load() * g_nsm);
    k_sort_segments_large<128, SEG_MID><<<large_grid, 128, SEG_MID * sizeof(uint32_t), s>>>(off, src_unsorted, src,
                                                                                          mid, nmid);
    return cudaGetLastError();
}

// bounds of the long segments listed in `big`
__global__ void k_long_bounds(const uint32_t* __restrict__ off, const int* __restrict__ big, int nbig,
                              uint32_t* __restrict__ b, uint32_t* __restrict__ e) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbig; i += gridDim.x * blockDim.x) {
        const int c = big[i];
        b[i] = off[c];
        e[i] = off[c + 1];
    }
}

size_t long_segments_temp(int nitems, int nlong, int end_bit) {
    size_t bytes = 0;
    cub::DeviceSegmentedRadixSort::SortKeys(nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr, nitems,
                                            nlong, (const uint32_t*)nullptr, (const uint32_t*)nullptr, 0, end_bit);
    return bytes;
}

cudaError_t sort_long_segments(void* tmp, size_t tmp_bytes, const uint32_t* off, const int* longs, int nlong,
                               const uint32_t* src_unsorted, uint32_t* src, int nitems, int end_bit, uint32_t* bounds,
                               cudaStream_t s) {
    if (nlong == 0) return cudaSuccess;
    k_long_bounds<<<grid_for(nlong, 256), 256, 0, s>>>(off, longs + 128, nlong, bounds, bounds + nlong);
    size_t bytes = tmp_bytes;
    return cub::DeviceSegmentedRadixSort::SortKeys(tmp, bytes, src_unsorted, src, nitems, nlong, bounds,
                                                   bounds + nlong, 0, end_bit, s);
}

}  // namespace fmmx
