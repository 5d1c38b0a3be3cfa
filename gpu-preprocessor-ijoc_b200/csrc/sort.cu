// Stable LSD radix sort of (uint64 key, int32 value) pairs.
//
// Replaces the reference's thrust::sort of (hash, id) tuples
// (rule_parallel_rows.cu:742-770, rule_parallel_columns.cu:958-975): with the
// input in ascending id order, a stable sort by key yields (key, id) order.
// Each 8-bit pass is three launches: per-tile digit histograms, one scan of
// the digit-major count table, and a stable scatter in which every warp ranks
// its keys with __match_any_sync and warps are ordered through shared
// counters.  Passes whose digit is constant across all keys are skipped
// (decided from one histogram readback per sort).
#include "sort.hpp"
#include "sort_kernels.cuh"

namespace gpp {

void radix_sort_pairs(uint64_t* keys, int32_t* vals, int64_t n, cudaStream_t s) {
  if (n <= 1) return;
  const int64_t tiles = (n + kTile - 1) / kTile;
  DBuf<unsigned long long> varies(1, s);
  varies.zero();
  GPP_LAUNCH(digit_variation, grid_stride_blocks(n), kThreads, 0, s, keys, n, varies.p);
  const uint64_t variation = read_scalar(varies.p);
  DBuf<uint64_t> k2(size_t(n), s);
  DBuf<int32_t> v2(size_t(n), s), counts(size_t(256 * tiles) + 1, s);
  uint64_t* ka = keys;
  int32_t* va = vals;
  uint64_t* kb = k2.p;
  int32_t* vb = v2.p;
  for (int pass = 0; pass < 8; ++pass) {
    if (((variation >> (8 * pass)) & 0xffu) == 0) continue;  // one digit for every key: the identity
    GPP_LAUNCH(digit_histogram, int(tiles), kThreads, 0, s, ka, n, 8 * pass, counts.p, tiles);
    exclusive_scan_i32(counts.p, counts.p, 256 * tiles, s);
    GPP_LAUNCH(digit_scatter, int(tiles), kThreads, 0, s, ka, va, n, 8 * pass, counts.p, tiles, kb, vb);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    check(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * size_t(n), cudaMemcpyDeviceToDevice, s), "sort copy keys");
    check(cudaMemcpyAsync(vals, va, sizeof(int32_t) * size_t(n), cudaMemcpyDeviceToDevice, s), "sort copy vals");
  }
}

}  // namespace gpp
