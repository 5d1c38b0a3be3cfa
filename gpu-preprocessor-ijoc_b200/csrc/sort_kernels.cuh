// Kernels of the stable LSD radix sort of (uint64 key, int32 value) pairs,
// shared by the pooled sort (sort.cu) and the fixed-scratch sort
// (sort_static.cu).  Each 8-bit pass is a per-tile digit histogram, an
// exclusive scan of the digit-major count table and a stable scatter in which
// every warp ranks its keys with __match_any_sync and warps are ordered
// through shared counters.
#pragma once

#include "common.cuh"

namespace gpp {

namespace {

constexpr int kTile = 2048;            // keys per block
constexpr int kItems = kTile / kThreads;

__global__ void digit_histogram(const uint64_t* __restrict__ keys, int64_t n, int shift, int32_t* __restrict__ counts,
                                int64_t tiles) {
  __shared__ int32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = int64_t(blockIdx.x) * kTile;
  for (int k = 0; k < kItems; ++k) {
    const int64_t i = base + int64_t(k) * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xff], 1);
  }
  __syncthreads();
  counts[int64_t(threadIdx.x) * tiles + blockIdx.x] = h[threadIdx.x];
}

// Digit presence over all 8 digit positions at once (for pass skipping).
__global__ void digit_presence(const uint64_t* __restrict__ keys, int64_t n, uint32_t* __restrict__ seen) {
  __shared__ uint32_t local[8 * 8];  // 8 passes x 256 bits
  if (threadIdx.x < 64) local[threadIdx.x] = 0;
  __syncthreads();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t k = keys[i];
    for (int pass = 0; pass < 8; ++pass) {
      const int d = int((k >> (8 * pass)) & 0xff);
      atomicOr(&local[pass * 8 + (d >> 5)], 1u << (d & 31));
    }
  }
  __syncthreads();
  if (threadIdx.x < 64 && local[threadIdx.x]) atomicOr(&seen[threadIdx.x], local[threadIdx.x]);
}

__global__ void digit_scatter(const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals, int64_t n, int shift,
                              const int32_t* __restrict__ offsets, int64_t tiles, uint64_t* __restrict__ out_keys,
                              int32_t* __restrict__ out_vals) {
  __shared__ int32_t running[256];
  __shared__ int32_t warp_digit_count[8][256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  running[threadIdx.x] = offsets[int64_t(threadIdx.x) * tiles + blockIdx.x];
  const int64_t base = int64_t(blockIdx.x) * kTile;
  for (int k = 0; k < kItems; ++k) {
    // Elements of this round: consecutive within the round, warp-major.
    const int64_t i = base + int64_t(k) * kThreads + threadIdx.x;
    const bool valid = i < n;
    const uint64_t key = valid ? keys[i] : 0;
    const int d = valid ? int((key >> shift) & 0xff) : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank_in_warp = __popc(peers & ((1u << lane) - 1u));
    for (int w = 0; w < 8; ++w) warp_digit_count[w][threadIdx.x] = 0;
    __syncthreads();
    if (valid && rank_in_warp == 0) warp_digit_count[warp][d] = __popc(peers);
    __syncthreads();
    int before = 0;
    if (valid)
      for (int w = 0; w < warp; ++w) before += warp_digit_count[w][d];
    if (valid) {
      const int64_t dst = int64_t(running[d]) + before + rank_in_warp;
      out_keys[dst] = key;
      out_vals[dst] = vals[i];
    }
    __syncthreads();
    // Advance the running offsets by this round's per-digit totals.
    int total = 0;
    for (int w = 0; w < 8; ++w) total += warp_digit_count[w][threadIdx.x];
    running[threadIdx.x] += total;
    __syncthreads();
  }
}

}  // namespace

}  // namespace gpp
