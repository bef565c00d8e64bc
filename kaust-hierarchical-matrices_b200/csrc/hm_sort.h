// hm_sort.h -- deterministic device sort / scan helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hm.h"

namespace hm {
// Stable ascending sort of n (key, value) pairs by the low key_bits bits of key.
hm_status sort_pairs_u32(uint32_t* keys, uint32_t* vals, int n, int key_bits, cudaStream_t stream);
// In-place exclusive scan; *d_total (device, may be null) receives the sum.
hm_status scan_exclusive(unsigned int* d_a, long long count, unsigned int* d_total,
                         cudaStream_t stream);
}  // namespace hm
