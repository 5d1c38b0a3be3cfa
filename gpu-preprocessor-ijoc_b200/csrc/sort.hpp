// Device sort primitive shared by the duplicate-detection rules.
#pragma once

#include "common.cuh"

namespace gpp {
// Stable sort of n (key, value) pairs by key, in place.
void radix_sort_pairs(uint64_t* keys, int32_t* vals, int64_t n, cudaStream_t s);
// The same sort with its scratch in a fixed device array (no allocation);
// n is at most GPP_SORT_STATIC_MAX_PAIRS.
void radix_sort_pairs_static(uint64_t* keys, int32_t* vals, int64_t n, cudaStream_t s);
}  // namespace gpp
