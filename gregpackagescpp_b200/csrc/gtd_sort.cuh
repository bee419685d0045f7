// Device scan and radix sort (sort.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gtd {

size_t scan_scratch_words(int64_t n);
int exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *scratch, cudaStream_t s,
                       uint64_t *launches);

size_t radix_scratch_words(int64_t n);
int radix_sort_u64(unsigned long long *keys, int32_t *vals, unsigned long long *keys_alt, int32_t *vals_alt,
                   int64_t n, int bits, uint32_t *scratch, cudaStream_t s, uint64_t *launches);

}  // namespace gtd
