// Directed, destination-segmented interaction lists.
//
// The walk emits mutual pairs, as the reference's recorder does
// (walk.rs:342-488). The evaluation kernels here are destination-owned (one
// CTA writes each cell's locals or each leaf's bodies, no atomics), so every
// mutual pair (a, b) becomes the two directed entries a->b and b->a, a leaf
// self pair one entry. Entries are radix-sorted by (dst, src), which makes the
// accumulation order, and therefore every result bit, independent of the
// order in which the walk's atomics appended pairs. A key is
// (dst << shift) | src with shift = the bit width of the cell count, so the
// sort runs over 2 * shift bits (32 for up to 65535 cells) instead of 64.
#include "common.cuh"
#include "kernels.h"

namespace fmmx {

template <typename K>
__global__ void k_expand_m2l(const uint2* __restrict__ pairs, int np, int shift, K* __restrict__ keys) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
        const uint2 pr = pairs[q];
        keys[2 * (size_t)q] = (K)(((uint64_t)pr.y << shift) | pr.x);      // a -> b
        keys[2 * (size_t)q + 1] = (K)(((uint64_t)pr.x << shift) | pr.y);  // b -> a
    }
}

// P2P: a self pair gives one entry; its second slot gets `sentinel`, a key
// above every valid one, so the valid entries are a prefix after sorting.
template <typename K>
__global__ void k_expand_p2p(const uint2* __restrict__ pairs, int np, int shift, const uint32_t* __restrict__ count,
                             uint64_t sentinel, K* __restrict__ keys,
                             unsigned long long* __restrict__ interactions) {
    unsigned long long local = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
        const uint2 pr = pairs[q];
        const unsigned long long ca = count[pr.x], cb = count[pr.y];
        if (pr.x == pr.y) {
            keys[2 * (size_t)q] = (K)(((uint64_t)pr.x << shift) | pr.x);
            keys[2 * (size_t)q + 1] = (K)sentinel;
            local += ca * (ca - 1);
        } else {
            keys[2 * (size_t)q] = (K)(((uint64_t)pr.y << shift) | pr.x);
            keys[2 * (size_t)q + 1] = (K)(((uint64_t)pr.x << shift) | pr.y);
            local += 2ull * ca * cb;
        }
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(interactions, local);
}

template <typename K>
__global__ void k_segments(const K* __restrict__ keys, int nkeys, int shift, uint32_t* __restrict__ seg_begin,
                           uint32_t* __restrict__ seg_end) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nkeys; i += gridDim.x * blockDim.x) {
        const uint32_t d = (uint32_t)((uint64_t)keys[i] >> shift);
        if (i == 0 || (uint32_t)((uint64_t)keys[i - 1] >> shift) != d) seg_begin[d] = i;
        if (i == nkeys - 1 || (uint32_t)((uint64_t)keys[i + 1] >> shift) != d) seg_end[d] = i + 1;
    }
}

template <typename K>
void launch_expand_m2l(unsigned grid, cudaStream_t s, const uint2* pairs, int np, int shift, K* keys) {
    k_expand_m2l<K><<<grid, 256, 0, s>>>(pairs, np, shift, keys);
}
template <typename K>
void launch_expand_p2p(unsigned grid, cudaStream_t s, const uint2* pairs, int np, int shift, const uint32_t* count,
                       uint64_t sentinel, K* keys, unsigned long long* interactions) {
    k_expand_p2p<K><<<grid, 256, 0, s>>>(pairs, np, shift, count, sentinel, keys, interactions);
}
template <typename K>
void launch_segments(unsigned grid, cudaStream_t s, const K* keys, int nkeys, int shift, uint32_t* seg_begin,
                     uint32_t* seg_end) {
    k_segments<K><<<grid, 256, 0, s>>>(keys, nkeys, shift, seg_begin, seg_end);
}
template void launch_expand_m2l<uint32_t>(unsigned, cudaStream_t, const uint2*, int, int, uint32_t*);
template void launch_expand_m2l<uint64_t>(unsigned, cudaStream_t, const uint2*, int, int, uint64_t*);
template void launch_expand_p2p<uint32_t>(unsigned, cudaStream_t, const uint2*, int, int, const uint32_t*, uint64_t,
                                          uint32_t*, unsigned long long*);
template void launch_expand_p2p<uint64_t>(unsigned, cudaStream_t, const uint2*, int, int, const uint32_t*, uint64_t,
                                          uint64_t*, unsigned long long*);
template void launch_segments<uint32_t>(unsigned, cudaStream_t, const uint32_t*, int, int, uint32_t*, uint32_t*);
template void launch_segments<uint64_t>(unsigned, cudaStream_t, const uint64_t*, int, int, uint32_t*, uint32_t*);

}  // namespace fmmx
