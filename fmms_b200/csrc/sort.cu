// Radix sorts used by the engine (Morton keys and the depth-first
// renumbering), via CUB's device radix sort. LSD radix sort is
// stable, so equal Morton keys keep ascending particle index: the tie rule of
// a stable sort_by_key (the reference's sort_unstable_by_key, tree.rs:130,
// leaves ties unspecified).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_segmented_radix_sort.cuh>

#include "sort.h"

namespace fmmx {

size_t sort_pairs_u64_u32_temp(int n, int end_bit) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, n, 0, end_bit);
    return bytes;
}

cudaError_t sort_pairs_u64_u32(void* tmp, size_t tmp_bytes, const uint64_t* kin, uint64_t* kout, const uint32_t* vin,
                               uint32_t* vout, int n, int end_bit, cudaStream_t s) {
    return cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kin, kout, vin, vout, n, 0, end_bit, s);
}

// Independent sorts of the segments [off[s], off[s+1]) (a forest of systems).
size_t sort_pairs_seg_temp(int n, int nseg, const uint64_t* off, int end_bit) {
    size_t bytes = 0;
    cub::DeviceSegmentedRadixSort::SortPairs(nullptr, bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                             (const uint32_t*)nullptr, (uint32_t*)nullptr, n, nseg, off, off + 1, 0,
                                             end_bit);
    return bytes;
}

cudaError_t sort_pairs_seg(void* tmp, size_t tmp_bytes, const uint64_t* kin, uint64_t* kout, const uint32_t* vin,
                           uint32_t* vout, int n, int nseg, const uint64_t* off, int end_bit, cudaStream_t s) {
    return cub::DeviceSegmentedRadixSort::SortPairs(tmp, tmp_bytes, kin, kout, vin, vout, n, nseg, off, off + 1, 0,
                                                    end_bit, s);
}

}  // namespace fmmx
