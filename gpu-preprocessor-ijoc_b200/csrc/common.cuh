// Shared device/host plumbing of the B200 presolve engine: error handling,
// the engine stream, stream-ordered buffers, launch accounting, and the
// deterministic scan / reduction primitives every kernel family uses.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../include/gpp.h"

namespace gpp {

using offset_t = gpp_offset;
constexpr int kThreads = 256;
constexpr int kEntryTile = 2048;    // stored entries per tile of the entry-parallel sweeps
constexpr int kShortRow = 8;      // rows of live length <= 8: one thread per row
constexpr int kLongRow = 1024;    // rows of live length > 1024: one block per row
constexpr int kNumSMs = 148;      // B200

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct InvalidArgument : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct LengthError : std::length_error {
  using std::length_error::length_error;
};

inline void check(cudaError_t e, const char* ctx) {
  if (e != cudaSuccess) throw CudaError(std::string(ctx) + ": " + cudaGetErrorString(e));
}

// An NVTX range over a scope (a presolve, a rule, a materialisation, a
// postsolve), for profilers that show them (ncu --nvtx); without a profiler
// attached the calls return at once.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Kernel launch counter (per host thread) for the benchmark's launch report.
uint64_t& launch_counter();
uint64_t& sync_counter();   // host waits on the engine stream, calling thread

// Optional per-launch timing (CUDA events on the launching stream) used by
// the benchmark's roofline report; off unless gpp_profile_enable(1).
bool profiling();
void profile_record(const char* name, double bytes, cudaEvent_t begin, cudaEvent_t end);
cudaEvent_t profile_event();
// The last recorded launch (-1 when not profiling), and a way to add bytes
// to it once they are known (a kernel whose output size is read back later).
int64_t profile_last();
void profile_add_bytes(int64_t record, double bytes);

#define GPP_LAUNCH_BYTES(kernel, bytes, grid, block, smem, stream, ...)             \
  do {                                                                              \
    if ((grid) > 0) {                                                               \
      cudaEvent_t gpp_ev0 = nullptr, gpp_ev1 = nullptr;                             \
      if (::gpp::profiling()) {                                                     \
        gpp_ev0 = ::gpp::profile_event();                                           \
        gpp_ev1 = ::gpp::profile_event();                                           \
        cudaEventRecord(gpp_ev0, (stream));                                         \
      }                                                                             \
      kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                   \
      ::gpp::check(cudaGetLastError(), #kernel);                                    \
      ++::gpp::launch_counter();                                                    \
      if (gpp_ev1) {                                                                \
        cudaEventRecord(gpp_ev1, (stream));                                         \
        ::gpp::profile_record(#kernel, double(bytes), gpp_ev0, gpp_ev1);            \
      }                                                                             \
    }                                                                               \
  } while (0)
#define GPP_LAUNCH(kernel, grid, block, smem, stream, ...) \
  GPP_LAUNCH_BYTES(kernel, 0.0, grid, block, smem, stream, __VA_ARGS__)

inline int blocks_for(int64_t n, int threads = kThreads) {
  const int64_t b = (n + threads - 1) / threads;
  return int(b < 1 ? 0 : (b > 2147483647 ? 2147483647 : b));
}
// Grid for grid-stride kernels: enough blocks to fill all 148 SMs several
// times over without launching more than the work needs.
inline int grid_stride_blocks(int64_t n, int threads = kThreads, int per_sm = 8) {
  const int64_t want = (n + threads - 1) / threads;
  const int64_t cap = int64_t(kNumSMs) * per_sm;
  return int(want < 1 ? 0 : (want < cap ? want : cap));
}

// Column bounds packed for the row sweeps: {l_j, u_j} in one 16-byte record,
// so a gathered column costs one memory sector instead of three (l, u and the
// keep mask).  A removed column holds one reserved NaN bit pattern in both
// fields; a kept column holds its bounds as they are (any value, NaN
// included), so the sweeps' arithmetic is unchanged.
constexpr unsigned long long kRemovedColumnBits = 0x7FF00000DEADC01EULL;
__device__ __forceinline__ bool removed_column(double2 b) {
  return static_cast<unsigned long long>(__double_as_longlong(b.x)) == kRemovedColumnBits;
}

// L2 residency hints for the row sweeps over A (activity summary, bound
// candidates).  Each stored entry gathers the 16-byte bound record of its
// column; a column's record is gathered once per entry of the column (about
// six times on the random family), while the CSR arrays are read exactly
// once.  At 25M nnz the records are 80 MB and the streamed CSR 360 MB, so
// with plain loads the stream pushes the records out of the 126 MB L2 and
// most gathers go to DRAM as 32-byte sectors.  Gathers therefore carry an
// L2 evict_last policy and streamed loads an evict_first policy that also
// skips L1 (PTX createpolicy + ld.global.nc.L2::cache_hint).  The hints only
// order evictions; the loaded values are the same.
struct L2Hints {
  uint64_t keep, stream;
};
__device__ __forceinline__ L2Hints l2_hints() {
  L2Hints h;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(h.keep));
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(h.stream));
  return h;
}
__device__ __forceinline__ double2 ld_keep(const double2* a, uint64_t pol) {
  double2 v;
  asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ int32_t ld_stream(const int32_t* a, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* a, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
  return v;
}

// Order-free max / min of doubles as single 64-bit integer reductions (RED,
// no value returned, nothing for the thread to wait on).  A double whose sign
// bit is clear orders like its bits read as a signed integer; one whose sign
// bit is set orders in reverse of its bits read as an unsigned integer, and
// every such pattern compares above every clear-sign pattern as unsigned and
// below it as signed.  So max = signed max for clear-sign values and unsigned
// min for set-sign values (min the other way round), which equals the
// load-and-CAS loop of the reference (rule_bound_strengthening.cu:299-335)
// for every input except the tie +0 / -0, where the CAS result depends on the
// arrival order and this one does not (max keeps +0, min keeps -0).  NaN
// values must not be passed.
__device__ __forceinline__ void red_max_f64(double* addr, double v) {
  const long long bits = __double_as_longlong(v);
  if (bits >= 0) atomicMax(reinterpret_cast<long long*>(addr), bits);
  else atomicMin(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(bits));
}
__device__ __forceinline__ void red_min_f64(double* addr, double v) {
  const long long bits = __double_as_longlong(v);
  if (bits >= 0) atomicMin(reinterpret_cast<long long*>(addr), bits);
  else atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(bits));
}

// Largest r in [lo, hi) with ptr[r] <= p: for a stored position p of a CSR
// matrix (ptr non-decreasing), the row that holds p (never an empty row).
__device__ __forceinline__ int row_of(const offset_t* ptr, int lo, int hi, offset_t p) {
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (ptr[mid] <= p) lo = mid; else hi = mid;
  }
  return lo;
}

// Warp-aggregated append: every lane of the warp must call it; lanes with
// `take` get consecutive slots (in lane order) from *counter, others get -1.
__device__ __forceinline__ int warp_append(int32_t* counter, bool take) {
  const unsigned mask = __ballot_sync(0xffffffffu, take);
  if (!mask) return -1;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  return take ? base + __popc(mask & ((1u << lane) - 1u)) : -1;
}

// Block-aggregated append: one atomic per block instead of one per warp (a
// per-warp atomic on one address serialises a grid-wide sweep).  Every
// thread of the block must call it the same number of times.
__device__ __forceinline__ int block_append(int32_t* counter, bool take) {
  __shared__ int warp_base[32];
  __shared__ int block_base;
  const unsigned mask = __ballot_sync(0xffffffffu, take);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_base[warp] = __popc(mask);
  __syncthreads();
  if (threadIdx.x == 0) {
    int total = 0;
    const int warps = (blockDim.x + 31) >> 5;
    for (int w = 0; w < warps; ++w) {
      const int c = warp_base[w];
      warp_base[w] = total;
      total += c;
    }
    block_base = total ? atomicAdd(counter, total) : 0;
  }
  __syncthreads();
  const int slot = take ? block_base + warp_base[warp] + __popc(mask & ((1u << lane) - 1u)) : -1;
  __syncthreads();
  return slot;
}

// ---------------------------------------------------------------------------
// Engine context: one stream (blocking w.r.t. the legacy default stream so
// caller work on stream 0 is ordered before ours), a stream-ordered memory
// pool that keeps its memory between calls, and a pinned status block.
struct Context {
  cudaStream_t stream = nullptr;
  int device = -1;
  cudaMemPool_t pool = nullptr;   // this context's own stream-ordered pool
  int32_t* host_status = nullptr;   // pinned, kStatusWords ints
  unsigned char* host_scalar = nullptr;   // pinned, 16 bytes for scalar readbacks
  unsigned long long* host_later = nullptr;   // pinned, one word read after a later wait
  cudaStream_t side = nullptr;
  // Scratch blocks this context freed on its own stream, by size class,
  // ready to be handed out again without a driver call (pool_alloc/free).
  std::unordered_map<size_t, std::vector<void*>> free_blocks;
  static constexpr int kStatusWords = 64;
  // A second stream for host-to-device copies that overlap the engine
  // stream's kernels (created on first use; ordered by events).
  cudaStream_t side_stream();
  Context();
  ~Context();
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  // Waits for the engine stream (`ctx` names the call site; while profiling,
  // each wait is recorded as "sync: <ctx>" with its host time).
  void sync(const char* ctx);
};
Context& ctx();

// Every engine device allocation: stream-ordered from the context's pool.
// A test hook (gpp_inject_alloc_failure) can make the k-th allocation after
// it was armed return cudaErrorMemoryAllocation instead, a host-side fake of
// an out-of-memory failure that touches no device state.
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s);
// Every engine device release (buffers of pool_alloc only).
void pool_free(void* p, cudaStream_t s);
void inject_alloc_failure(int64_t after);

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  DBuf() = default;
  explicit DBuf(size_t count, cudaStream_t stream = nullptr) { alloc(count, stream); }
  void alloc(size_t count, cudaStream_t stream = nullptr) {
    release();
    s = stream ? stream : ctx().stream;
    n = count;
    if (count) check(pool_alloc(reinterpret_cast<void**>(&p), count * sizeof(T), s), "cudaMallocFromPoolAsync");
  }
  void release() {
    if (p) pool_free(p, s);
    p = nullptr;
    n = 0;
  }
  T* release_ownership() {
    T* q = p;
    p = nullptr;
    n = 0;
    return q;
  }
  ~DBuf() { release(); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(std::exchange(o.p, nullptr)), n(std::exchange(o.n, 0)), s(o.s) {}
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = std::exchange(o.p, nullptr);
      n = std::exchange(o.n, 0);
      s = o.s;
    }
    return *this;
  }
  T* get() const { return p; }
  void zero() {
    if (n) check(cudaMemsetAsync(p, 0, n * sizeof(T), s), "cudaMemsetAsync");
  }
  void copy_from(const T* src, size_t count) {
    if (count) check(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyDeviceToDevice, s), "copy d2d");
  }
};

template <class T>
T* dalloc(size_t count) {
  T* p = nullptr;
  if (count)
    check(pool_alloc(reinterpret_cast<void**>(&p), count * sizeof(T), ctx().stream), "cudaMallocFromPoolAsync");
  return p;
}
inline void dfree(void* p) {
  if (p) pool_free(p, ctx().stream);
}

template <class T>
std::vector<T> to_host(const T* d, size_t count) {
  std::vector<T> h(count);
  if (count) {
    check(cudaMemcpyAsync(h.data(), d, count * sizeof(T), cudaMemcpyDeviceToHost, ctx().stream), "d2h");
    ctx().sync("d2h sync");
  }
  return h;
}
// Two arrays in one wait.
template <class T, class U>
std::pair<std::vector<T>, std::vector<U>> to_host2(const T* a, size_t na, const U* b, size_t nb) {
  std::vector<T> ha(na);
  std::vector<U> hb(nb);
  if (na) check(cudaMemcpyAsync(ha.data(), a, na * sizeof(T), cudaMemcpyDeviceToHost, ctx().stream), "d2h");
  if (nb) check(cudaMemcpyAsync(hb.data(), b, nb * sizeof(U), cudaMemcpyDeviceToHost, ctx().stream), "d2h");
  if (na || nb) ctx().sync("d2h sync");
  return {std::move(ha), std::move(hb)};
}
template <class T>
T read_scalar(const T* d, const char* where = __builtin_FUNCTION()) {
  // Through the context's pinned block: a pageable destination would make
  // the copy go through a staging buffer.
  static_assert(sizeof(T) <= 8, "scalar");
  auto& c = ctx();
  check(cudaMemcpyAsync(c.host_scalar, d, sizeof(T), cudaMemcpyDeviceToHost, c.stream), "d2h scalar");
  c.sync(where);
  T v;
  std::memcpy(&v, c.host_scalar, sizeof(T));
  return v;
}
// Two scalars (say the totals of two scans) with one wait.
template <class T, class U>
std::pair<T, U> read_scalars(const T* a, const U* b, const char* where = __builtin_FUNCTION()) {
  static_assert(sizeof(T) <= 8 && sizeof(U) <= 8, "scalar");
  auto& c = ctx();
  unsigned char* h = c.host_scalar;
  check(cudaMemcpyAsync(h, a, sizeof(T), cudaMemcpyDeviceToHost, c.stream), "d2h scalar");
  check(cudaMemcpyAsync(h + 8, b, sizeof(U), cudaMemcpyDeviceToHost, c.stream), "d2h scalar");
  c.sync(where);
  T va;
  U vb;
  std::memcpy(&va, h, sizeof(T));
  std::memcpy(&vb, h + 8, sizeof(U));
  return {va, vb};
}

// Status block: device ints zeroed per use, read back with one copy.
struct Status {
  int32_t* d = nullptr;
  Status();
  ~Status();
  void clear(int words = Context::kStatusWords);
  // `where` (the calling function) labels the wait in the benchmark's profile.
  const int32_t* read(int words = Context::kStatusWords, const char* where = __builtin_FUNCTION());
};

// ---------------------------------------------------------------------------
// Scans (decoupled into three small kernels; deterministic, any length).
// exclusive prefix sum of in[0..n) into out[0..n]; out[n] = total.  out may
// alias in for n+1-sized storage only when in has n+1 slots.
void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s);
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);

// Canonical deterministic sum (chunks of 2048, 256-thread halving tree, chunk
// totals added in order on the host).  Returns the value on the host.
double det_sum(const double* v, int64_t n, cudaStream_t s);
// det_sum of a length-n vector that is zero except at the given (index,
// value) entries, evaluated on the host in the same association: the +0.0
// terms of the dense form are identities, so only the entries are needed.
double det_sum_sparse(std::vector<std::pair<int64_t, double>> entries);

struct ProfileSummary {
  std::string name;
  int64_t launches;
  double ms;
  double bytes;
};
void profile_enable(bool on);
void profile_sync(const char* label, double ms);
std::vector<ProfileSummary> profile_summary();

// Thread-local error message for the C ABI.
void set_last_error(const std::string& s);

}  // namespace gpp
