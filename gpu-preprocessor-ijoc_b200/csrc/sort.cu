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

#include <mutex>
#include <vector>

namespace gpp {

namespace {

// Small inputs (most sorts of a presolve round: the winners of one rule,
// the hashes of the few changed rows) take one block instead of up to eight
// three-launch passes and a readback: a bitonic network over (key, original
// position) in shared memory.  The order on (key, position) is total, so the
// result is exactly the stable sort's.
constexpr int kBlockSortMax = 4096;
constexpr int kBlockSortThreads = 1024;

__global__ void __launch_bounds__(kBlockSortThreads) block_sort_pairs(uint64_t* keys, int32_t* vals, int n, int size) {
  extern __shared__ unsigned char block_sort_smem[];
  auto* k = reinterpret_cast<uint64_t*>(block_sort_smem);
  auto* pos = reinterpret_cast<int32_t*>(k + size);
  auto* v = pos + size;
  for (int i = threadIdx.x; i < size; i += blockDim.x) {
    const bool in = i < n;
    k[i] = in ? keys[i] : ~0ull;
    pos[i] = in ? i : 0x7fffffff;
    v[i] = in ? vals[i] : 0;
  }
  __syncthreads();
  for (int width = 2; width <= size; width <<= 1) {
    for (int stride = width >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < size; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & width) == 0;
          const bool greater = k[i] > k[j] || (k[i] == k[j] && pos[i] > pos[j]);
          if (greater == up) {
            const uint64_t tk = k[i]; k[i] = k[j]; k[j] = tk;
            const int32_t tp = pos[i]; pos[i] = pos[j]; pos[j] = tp;
            const int32_t tv = v[i]; v[i] = v[j]; v[j] = tv;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    keys[i] = k[i];
    vals[i] = v[i];
  }
}

}  // namespace

void radix_sort_pairs(uint64_t* keys, int32_t* vals, int64_t n, cudaStream_t s) {
  if (n <= 1) return;
  if (n <= kBlockSortMax) {
    int size = 2;
    while (size < n) size <<= 1;
    const size_t smem = size_t(size) * (sizeof(uint64_t) + 2 * sizeof(int32_t));
    // The shared-memory limit is a per-device function attribute: set it once
    // per device, with that device current.
    static std::mutex mu;
    static std::vector<bool> configured;
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    {
      std::lock_guard<std::mutex> lock(mu);
      if (size_t(dev) >= configured.size()) configured.resize(size_t(dev) + 1, false);
      if (!configured[size_t(dev)]) {
        check(cudaFuncSetAttribute(block_sort_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(kBlockSortMax * (sizeof(uint64_t) + 2 * sizeof(int32_t)))),
              "block_sort_pairs smem");
        configured[size_t(dev)] = true;
      }
    }
    GPP_LAUNCH(block_sort_pairs, 1, kBlockSortThreads, smem, s, keys, vals, int(n), size);
    return;
  }
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
