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

// Which digit positions vary (for pass skipping): the OR over all keys of
// key ^ keys[0].  A byte of it is zero exactly when every key has the same
// digit there, and that pass is the identity.  One register OR per thread,
// a warp reduction, one atomic per warp per half.
__global__ void digit_variation(const uint64_t* __restrict__ keys, int64_t n, unsigned long long* __restrict__ out) {
  const uint64_t first = keys[0];
  uint64_t acc = 0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    acc |= keys[i] ^ first;
  const uint32_t lo = __reduce_or_sync(0xffffffffu, uint32_t(acc));
  const uint32_t hi = __reduce_or_sync(0xffffffffu, uint32_t(acc >> 32));
  if ((threadIdx.x & 31) == 0 && (lo | hi)) atomicOr(out, (uint64_t(hi) << 32) | lo);
}

// Stable scatter of one tile: the tile's keys are first ranked into a
// digit-sorted order in shared memory (warp ranks from __match_any_sync,
// warps ordered through shared counters, rounds in tile order), then written
// out so consecutive threads store consecutive slots of one digit's run:
// coalesced runs instead of one sector per key.
__global__ void __launch_bounds__(kThreads)
digit_scatter(const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals, int64_t n, int shift,
              const int32_t* __restrict__ offsets, int64_t tiles, uint64_t* __restrict__ out_keys,
              int32_t* __restrict__ out_vals) {
  __shared__ int32_t running[256];      // next tile-local slot of each digit
  __shared__ int32_t digit_start[256];  // tile-local start of each digit's run
  __shared__ int32_t global_start[256]; // global position of the run's first slot
  __shared__ int32_t warp_digit_count[8][256];
  __shared__ uint64_t local_keys[kTile];
  __shared__ int32_t local_vals[kTile];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = int64_t(blockIdx.x) * kTile;
  const int tile_n = int(min(int64_t(kTile), n - base));
  // The scanned digit-major table holds this tile's run start of every
  // digit; the next entry (the same digit's next tile, or the next digit's
  // first tile) minus it is the tile's count of that digit, so no recount.
  const int64_t at = int64_t(threadIdx.x) * tiles + blockIdx.x;
  const int32_t start_d = offsets[at];
  const int32_t count_d = offsets[at + 1] - start_d;
  global_start[threadIdx.x] = start_d;
  {
    // Exclusive scan of the 256 tile counts, one digit per thread.
    __shared__ int32_t warp_total[8];
    int32_t incl = count_d;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int32_t peer = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += peer;
    }
    if (lane == 31) warp_total[warp] = incl;
    __syncthreads();
    int32_t before = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) before += w < warp ? warp_total[w] : 0;
    digit_start[threadIdx.x] = before + incl - count_d;
    running[threadIdx.x] = before + incl - count_d;
  }
  __syncthreads();
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
    if (valid) {
      int before = 0;
      for (int w = 0; w < warp; ++w) before += warp_digit_count[w][d];
      const int slot = running[d] + before + rank_in_warp;
      local_keys[slot] = key;
      local_vals[slot] = vals[i];
    }
    __syncthreads();
    int total = 0;
    for (int w = 0; w < 8; ++w) total += warp_digit_count[w][threadIdx.x];
    running[threadIdx.x] += total;
    __syncthreads();
  }
  // Write the digit-sorted tile: slot q of digit d goes to global_start[d] +
  // (q - digit_start[d]).
  for (int q = threadIdx.x; q < tile_n; q += kThreads) {
    const uint64_t key = local_keys[q];
    const int d = int((key >> shift) & 0xff);
    const int64_t dst = int64_t(global_start[d]) + (q - digit_start[d]);
    out_keys[dst] = key;
    out_vals[dst] = local_vals[q];
  }
}

}  // namespace

}  // namespace gpp
