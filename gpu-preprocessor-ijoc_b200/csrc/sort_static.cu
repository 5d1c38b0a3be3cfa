// Stable radix sort of (uint64 key, int32 value) pairs that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they want to sort:
// code that runs under a custom or arena allocator that owns all of the
// device's memory, code that has promised its host application a fixed
// footprint, and code running while an allocation would have to wait for the
// pool to be trimmed.  For them this sort keeps its whole scratch (the
// ping-pong copy of the pairs and the per-tile digit count table) in one
// file-scope device array of a fixed size, so a call issues kernel launches on
// the caller's stream and nothing else: no cudaMalloc, no cudaFree, no pool,
// no host readback.
//
// Differences from the pooled sort (sort.cu), none of which changes the
// output: all eight 8-bit passes always run (there is no readback to decide
// which passes are constant), and eight passes bring the pairs back into the
// caller's buffers, so no final copy is needed.  A stable sort's output is
// unique, so both sorts return the same pairs.
//
// Every call shares the one array: calls whose work overlaps on the GPU
// (different streams, or different host threads without ordering between
// them) race on it and give wrong results.  Nothing in the array has to start
// at zero: each pass writes every count it later reads.
//
// Set-up.  CUDA loads a library's device code lazily, so the first call on a
// device loads this module, and with it the fixed array: that load is the one
// device allocation this entry point ever causes.  The same first call looks
// up the array's device address (cudaGetSymbolAddress) with the device
// current and keeps it for the rest of the process.  Any call does this, even
// one with n <= 1, so a caller can warm a device up with an empty sort before
// its arena takes the device's memory and before any stream capture.  A
// cudaDeviceReset unloads the module; the kept address is then stale, so this
// entry point must not be used on a device after it has been reset.
#include <mutex>
#include <stdexcept>
#include <string>

#include "gpp.h"
#include "sort.hpp"
#include "sort_kernels.cuh"

namespace gpp {

namespace {

constexpr int64_t kStaticPairs = GPP_SORT_STATIC_MAX_PAIRS;
constexpr int64_t kStaticTiles = (kStaticPairs + kTile - 1) / kTile;
constexpr int64_t kStaticCounts = 256 * kStaticTiles + 1;   // digit-major table and its total
constexpr size_t kKeysOffset = 0;
constexpr size_t kValsOffset = kKeysOffset + sizeof(uint64_t) * size_t(kStaticPairs);
constexpr size_t kCountsOffset = kValsOffset + sizeof(int32_t) * size_t(kStaticPairs);
constexpr size_t kScratchBytes = kCountsOffset + sizeof(int32_t) * size_t(kStaticCounts);
static_assert(kValsOffset % 256 == 0 && kCountsOffset % 256 == 0, "scratch sections stay 256-byte aligned");

// 8 MiB of keys + 4 MiB of values + 512 KiB of counts at the maximum size.
static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of this device's copy of g_sort_scratch, looked up once per
// device with that device current.
unsigned char* scratch_for_current_device() {
  int dev = -1;
  check(cudaGetDevice(&dev), "sort_pairs_static: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("sort_pairs_static: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    check(cudaGetSymbolAddress(&p, g_sort_scratch), "sort_pairs_static: cudaGetSymbolAddress");
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  return g_scratch_ptr[dev];
}

// In-place exclusive scan of the digit-major count table by one block of
// 1024 threads: thread t owns a contiguous chunk, chunk sums are scanned in
// shared memory.  The table holds at most 256 x 512 counts.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) scan_counts_one_block(int32_t* __restrict__ counts, int64_t n) {
  __shared__ int32_t sm[kScanThreads];
  const int64_t chunk = (n + kScanThreads - 1) / kScanThreads;
  const int64_t begin = int64_t(threadIdx.x) * chunk;
  const int64_t end = begin + chunk < n ? begin + chunk : n;
  int32_t local = 0;
  for (int64_t i = begin; i < end; ++i) local += counts[i];
  sm[threadIdx.x] = local;
  __syncthreads();
  for (int off = 1; off < kScanThreads; off <<= 1) {
    const int32_t t = threadIdx.x >= unsigned(off) ? sm[threadIdx.x - off] : 0;
    __syncthreads();
    sm[threadIdx.x] += t;
    __syncthreads();
  }
  int32_t run = threadIdx.x ? sm[threadIdx.x - 1] : 0;
  for (int64_t i = begin; i < end; ++i) {
    const int32_t v = counts[i];
    counts[i] = run;
    run += v;
  }
  if (threadIdx.x == kScanThreads - 1) counts[n] = sm[kScanThreads - 1];   // the total, read by the scatter
}

void launched(const char* what) {
  ++launch_counter();
  check(cudaGetLastError(), what);
}

}  // namespace

void radix_sort_pairs_static(uint64_t* keys, int32_t* vals, int64_t n, cudaStream_t s) {
  if (n < 0) throw std::invalid_argument("sort_pairs_static: negative pair count");
  if (n > kStaticPairs)
    throw std::length_error("sort_pairs_static: " + std::to_string(n) + " pairs exceed the fixed scratch capacity of " +
                            std::to_string(kStaticPairs) + " pairs; use gpp_sort_pairs");
  // Set-up first, so that any call, even an empty one, loads the module and
  // looks up the array's address.
  unsigned char* scratch = scratch_for_current_device();
  if (n <= 1) return;
  if (!keys || !vals) throw std::invalid_argument("sort_pairs_static: null key or value pointer");
  auto* kb = reinterpret_cast<uint64_t*>(scratch + kKeysOffset);
  auto* vb = reinterpret_cast<int32_t*>(scratch + kValsOffset);
  auto* counts = reinterpret_cast<int32_t*>(scratch + kCountsOffset);
  const int64_t tiles = (n + kTile - 1) / kTile;
  uint64_t* ka = keys;
  int32_t* va = vals;
  for (int pass = 0; pass < 8; ++pass) {
    digit_histogram<<<int(tiles), kThreads, 0, s>>>(ka, n, 8 * pass, counts, tiles);
    launched("sort_pairs_static: digit_histogram");
    scan_counts_one_block<<<1, kScanThreads, 0, s>>>(counts, 256 * tiles);
    launched("sort_pairs_static: scan_counts_one_block");
    digit_scatter<<<int(tiles), kThreads, 0, s>>>(ka, va, n, 8 * pass, counts, tiles, kb, vb);
    launched("sort_pairs_static: digit_scatter");
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  // Eight passes: the sorted pairs are back in the caller's buffers.
}

}  // namespace gpp
