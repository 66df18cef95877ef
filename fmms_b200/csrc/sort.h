#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace fmmx {
size_t sort_pairs_u64_u32_temp(int n, int end_bit);
cudaError_t sort_pairs_u64_u32(void* tmp, size_t tmp_bytes, const uint64_t* kin, uint64_t* kout, const uint32_t* vin,
                               uint32_t* vout, int n, int end_bit, cudaStream_t s);
size_t sort_pairs_seg_temp(int n, int nseg, const uint64_t* off, int end_bit);
cudaError_t sort_pairs_seg(void* tmp, size_t tmp_bytes, const uint64_t* kin, uint64_t* kout, const uint32_t* vin,
                           uint32_t* vout, int n, int nseg, const uint64_t* off, int end_bit, cudaStream_t s);
}  // namespace fmmx
