// Engine context, status block, scans and the canonical deterministic sum.
#include "common.cuh"

#include <atomic>
#include <cstdlib>

#include <algorithm>
#include <chrono>
#include <string>
#include <memory>
#include <mutex>
#include <unordered_map>

namespace gpp {

uint64_t& launch_counter() {
  static thread_local uint64_t count = 0;
  return count;
}
uint64_t& sync_counter() {
  static thread_local uint64_t n = 0;
  return n;
}

Context::Context() {
  check(cudaGetDevice(&device), "cudaGetDevice");
  // Blocking stream: implicitly ordered after work the caller queued on the
  // legacy default stream, as the reference's synchronous API assumes.
  check(cudaStreamCreateWithFlags(&stream, cudaStreamDefault), "cudaStreamCreate");
  // A pool of this context alone: with one pool per host thread, the batched
  // form's workers neither share a pool lock nor get ordered after each other
  // by block reuse across their streams.
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
  uint64_t keep = UINT64_MAX;  // keep freed blocks in the pool between presolve calls
  check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool threshold");
  check(cudaMallocHost(reinterpret_cast<void**>(&host_status), sizeof(int32_t) * kStatusWords),
        "cudaMallocHost status");
  check(cudaMallocHost(reinterpret_cast<void**>(&host_scalar), 16), "cudaMallocHost scalar");
  check(cudaMallocHost(reinterpret_cast<void**>(&host_later), sizeof(unsigned long long)), "cudaMallocHost later");
}

void Context::sync(const char* label) {
  ++sync_counter();
  if (!profiling()) {
    check(cudaStreamSynchronize(stream), label);
    return;
  }
  const auto t0 = std::chrono::steady_clock::now();
  check(cudaStreamSynchronize(stream), label);
  profile_sync(label, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
}

Context::~Context() {
  if (host_status) cudaFreeHost(host_status);
  if (host_scalar) cudaFreeHost(host_scalar);
  if (host_later) cudaFreeHost(host_later);
  if (side) cudaStreamDestroy(side);
  if (stream) cudaStreamDestroy(stream);
}

cudaStream_t Context::side_stream() {
  if (!side) check(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking), "cudaStreamCreate side");
  return side;
}

Context& ctx() {
  // One context per host thread and device (the reference's contract is one
  // presolve per host thread on the current device).
  // Never destroyed: the stream and pinned block stay valid until process
  // exit, so buffers released during thread-exit destruction can still be
  // returned to the stream-ordered pool.
  static thread_local std::vector<Context*>* per_device = new std::vector<Context*>();
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (size_t(dev) >= per_device->size()) per_device->resize(size_t(dev) + 1, nullptr);
  if (!(*per_device)[size_t(dev)]) (*per_device)[size_t(dev)] = new Context();
  return *(*per_device)[size_t(dev)];
}

namespace {
std::atomic<int64_t> g_alloc_countdown{-1};   // < 0: no failure armed
}  // namespace

void inject_alloc_failure(int64_t after) { g_alloc_countdown.store(after < 0 ? -1 : after); }

// Host-side reuse of scratch blocks.  A presolve allocates and frees a few
// thousand scratch buffers, each a cudaMallocFromPoolAsync / cudaFreeAsync
// pair of driver calls on the host's critical path between launches.  Blocks
// are rounded up to a size class (at most 25% over) and a block its own
// context frees on that context's stream goes to the context's free list; the
// next request of that class on that stream takes it back with no driver
// call.  Reuse is safe without events: everything on one stream runs in issue
// order, so a kernel that gets the block runs after every kernel that used it.
// A block freed by another thread or on another stream goes back to the pool.
// At most kCachedCap bytes are held this way across all contexts; past that a
// freed block goes back to the pool.  GPP_ALLOC_CACHE=0 turns the reuse off.
namespace {
struct HandedOut {
  size_t bytes;
  const Context* owner;
};
std::mutex g_blocks_mu;
std::unordered_map<void*, HandedOut>* g_blocks = new std::unordered_map<void*, HandedOut>();   // never destroyed
std::atomic<int64_t> g_cached_bytes{0};
constexpr int64_t kCachedCap = int64_t(8) << 30;

bool alloc_cache_on() {
  static const bool on = [] {
    const char* e = std::getenv("GPP_ALLOC_CACHE");
    return !(e && e[0] == '0');
  }();
  return on;
}
size_t size_class(size_t bytes) {
  if (bytes <= 256) return 256;
  const int high = 63 - __builtin_clzll(uint64_t(bytes));
  const size_t grain = size_t(1) << std::max(8, high - 2);
  return (bytes + grain - 1) / grain * grain;
}
}  // namespace

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s) {
  if (g_alloc_countdown.load(std::memory_order_relaxed) >= 0) {
    int64_t left = g_alloc_countdown.load();
    while (left >= 0 && !g_alloc_countdown.compare_exchange_weak(left, left - 1)) {
    }
    if (left == 0) {
      *p = nullptr;
      return cudaErrorMemoryAllocation;
    }
  }
  Context& c = ctx();
  if (!alloc_cache_on()) return cudaMallocFromPoolAsync(p, bytes, c.pool, s);
  const size_t cls = size_class(bytes);
  if (s == c.stream) {
    auto it = c.free_blocks.find(cls);
    if (it != c.free_blocks.end() && !it->second.empty()) {
      *p = it->second.back();
      it->second.pop_back();
      g_cached_bytes.fetch_sub(int64_t(cls), std::memory_order_relaxed);
      std::lock_guard<std::mutex> lock(g_blocks_mu);
      (*g_blocks)[*p] = HandedOut{cls, &c};
      return cudaSuccess;
    }
  }
  const cudaError_t e = cudaMallocFromPoolAsync(p, cls, c.pool, s);
  if (e == cudaSuccess) {
    std::lock_guard<std::mutex> lock(g_blocks_mu);
    (*g_blocks)[*p] = HandedOut{cls, &c};
  }
  return e;
}

void pool_free(void* p, cudaStream_t s) {
  if (!p) return;
  if (alloc_cache_on()) {
    HandedOut b{0, nullptr};
    {
      std::lock_guard<std::mutex> lock(g_blocks_mu);
      auto it = g_blocks->find(p);
      if (it != g_blocks->end()) {
        b = it->second;
        g_blocks->erase(it);
      }
    }
    Context& c = ctx();
    if (b.owner == &c && s == c.stream &&
        g_cached_bytes.fetch_add(int64_t(b.bytes), std::memory_order_relaxed) + int64_t(b.bytes) <= kCachedCap) {
      c.free_blocks[b.bytes].push_back(p);
      return;
    }
    if (b.owner == &c && s == c.stream) g_cached_bytes.fetch_sub(int64_t(b.bytes), std::memory_order_relaxed);
  }
  cudaFreeAsync(p, s);
}

Status::Status() {
  check(pool_alloc(reinterpret_cast<void**>(&d), sizeof(int32_t) * Context::kStatusWords, ctx().stream),
        "status alloc");
}
Status::~Status() { if (d) pool_free(d, ctx().stream); }
void Status::clear(int words) {
  check(cudaMemsetAsync(d, 0, sizeof(int32_t) * size_t(words), ctx().stream), "status clear");
}
const int32_t* Status::read(int words, const char* where) {
  auto& c = ctx();
  check(cudaMemcpyAsync(c.host_status, d, sizeof(int32_t) * size_t(words), cudaMemcpyDeviceToHost, c.stream),
        "status read");
  c.sync(where);
  return c.host_status;
}

namespace {
constexpr int kScanTile = 2048;  // 256 threads x 8 consecutive items
constexpr int kScanWarps = kThreads / 32;

// Block-wide sum of one value per thread (integers: any order); every
// thread gets the result.  Contains __syncthreads.
template <class T>
__device__ __forceinline__ T block_total(T v, T* warp_sums) {
#pragma unroll
  for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = v;
  __syncthreads();
  T t = 0;
#pragma unroll
  for (int w = 0; w < kScanWarps; ++w) t += warp_sums[w];
  __syncthreads();
  return t;
}

// Block-wide exclusive scan of one value per thread, in thread order.
// Contains __syncthreads.
template <class T>
__device__ __forceinline__ T block_exclusive(T v, T* warp_sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T peer = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += peer;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  T before = 0;
#pragma unroll
  for (int w = 0; w < kScanWarps; ++w) before += w < warp ? warp_sums[w] : T(0);
  __syncthreads();
  return before + incl - v;
}

template <class T>
__global__ void __launch_bounds__(kThreads) tile_reduce(const T* __restrict__ in, int64_t n, T* __restrict__ tile_sums) {
  __shared__ T warp_sums[kScanWarps];
  const int64_t base = int64_t(blockIdx.x) * kScanTile;
  T acc = 0;
#pragma unroll
  for (int k = 0; k < kScanTile / kThreads; ++k) {
    const int64_t i = base + int64_t(k) * kThreads + threadIdx.x;
    if (i < n) acc += in[i];
  }
  acc = block_total(acc, warp_sums);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = acc;
}

// Each block scans its tile (thread t owns 8 consecutive items) from the sum
// of all earlier tiles, which it adds up itself; the last block writes the
// total to out[n].  `in` and `out` may alias: a thread reads its own items
// before it writes them, and no thread touches another's.
template <class T>
__global__ void __launch_bounds__(kThreads) tile_scan(const T* in, int64_t n, const T* __restrict__ tile_sums,
                                                     T* out) {
  __shared__ T warp_sums[kScanWarps];
  T offset = 0;
  for (int k = threadIdx.x; k < int(blockIdx.x); k += kThreads) offset += tile_sums[k];
  offset = block_total(offset, warp_sums);
  const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * 8;
  T v[8];
  T local = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    v[k] = base + k < n ? in[base + k] : T(0);
    local += v[k];
  }
  T run = offset + block_exclusive(local, warp_sums);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == kThreads - 1) out[n] = run;
}

// Scan of up to kSmallScan items in one block of 1024 threads: thread t owns
// a run of consecutive items; the runs' sums are scanned across the block by
// warp shuffles and one shared round of warp totals.  `in` and `out` may
// alias (each thread reads its items before writing them).
constexpr int kSmallScanThreads = 1024;
constexpr int64_t kSmallScan = 32 * kSmallScanThreads;

template <class T>
__global__ void __launch_bounds__(kSmallScanThreads) small_scan(const T* in, int64_t n, T* out) {
  __shared__ T warp_sums[kSmallScanThreads / 32];
  const int64_t per = (n + kSmallScanThreads - 1) / kSmallScanThreads;
  const int64_t begin = int64_t(threadIdx.x) * per;
  const int64_t end = min(n, begin + per);
  T local = 0;
  for (int64_t i = begin; i < end; ++i) local += in[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = local;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T peer = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += peer;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  T before = 0;
  for (int w = 0; w < warp; ++w) before += warp_sums[w];
  T run = before + incl - local;
  for (int64_t i = begin; i < end; ++i) {
    const T v = in[i];
    out[i] = run;
    run += v;
  }
  if (threadIdx.x == kSmallScanThreads - 1) out[n] = before + incl;
}

// Exclusive scan of n items into out[0..n], out[n] the total: one launch up
// to kSmallScan items, two above.
template <class T>
void exclusive_scan(const T* in, T* out, int64_t n, cudaStream_t s) {
  if (n <= 0) {
    check(cudaMemsetAsync(out, 0, sizeof(T), s), "scan empty");
    return;
  }
  if (n <= kSmallScan) {
    GPP_LAUNCH(small_scan<T>, 1, kSmallScanThreads, 0, s, in, n, out);
    return;
  }
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  DBuf<T> sums(size_t(tiles), s);
  GPP_LAUNCH(tile_reduce<T>, int(tiles), kThreads, 0, s, in, n, sums.p);
  GPP_LAUNCH(tile_scan<T>, int(tiles), kThreads, 0, s, in, n, sums.p, out);
}

__global__ void det_sum_chunks(const double* __restrict__ v, int64_t n, double* __restrict__ out) {
  __shared__ double sm[kThreads];
  const int64_t base = int64_t(blockIdx.x) * 2048;
  double acc = 0.0;
  for (int64_t k = base + threadIdx.x; k < n && k < base + 2048; k += kThreads) acc += v[k];
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < unsigned(h)) sm[threadIdx.x] = sm[threadIdx.x] + sm[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sm[0];
}
}  // namespace

void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s) {
  exclusive_scan<int32_t>(in, out, n, s);
}
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
  exclusive_scan<int64_t>(in, out, n, s);
}

double det_sum(const double* v, int64_t n, cudaStream_t s) {
  if (n <= 0) return 0.0;
  const int64_t chunks = (n + 2047) / 2048;
  DBuf<double> part(size_t(chunks), s);
  GPP_LAUNCH(det_sum_chunks, int(chunks), kThreads, 0, s, v, n, part.p);
  std::vector<double> h(static_cast<size_t>(chunks));
  check(cudaMemcpyAsync(h.data(), part.p, sizeof(double) * size_t(chunks), cudaMemcpyDeviceToHost, s), "det_sum d2h");
  ++sync_counter();
  check(cudaStreamSynchronize(s), "det_sum sync");
  double total = 0.0;
  for (double x : h) total += x;
  return total;
}

double det_sum_sparse(std::vector<std::pair<int64_t, double>> entries) {
  std::sort(entries.begin(), entries.end(),
            [](const std::pair<int64_t, double>& a, const std::pair<int64_t, double>& b) { return a.first < b.first; });
  double total = 0.0;
  size_t k = 0;
  while (k < entries.size()) {
    const int64_t chunk = entries[k].first / 2048;
    double slot[kThreads] = {};
    for (; k < entries.size() && entries[k].first / 2048 == chunk; ++k)
      slot[entries[k].first % kThreads] += entries[k].second;
    for (int h = kThreads / 2; h > 0; h >>= 1)
      for (int t = 0; t < h; ++t) slot[t] = slot[t] + slot[t + h];
    total += slot[0];
  }
  return total;
}

namespace {
thread_local std::string g_last_error;

struct ProfileRecord {
  std::string name;
  double bytes;
  cudaEvent_t begin, end;   // null for a host wait, whose host time is host_ms
  double host_ms;
};
struct ProfileState {
  bool on = false;
  std::vector<ProfileRecord> records;
  std::vector<cudaEvent_t> pool;
  size_t next = 0;
};
ProfileState& profile_state() {
  static thread_local ProfileState* p = new ProfileState;  // never destroyed (see ctx())
  return *p;
}
}  // namespace

bool profiling() { return profile_state().on; }
cudaEvent_t profile_event() {
  auto& p = profile_state();
  if (p.next == p.pool.size()) {
    cudaEvent_t e;
    check(cudaEventCreate(&e), "cudaEventCreate");
    p.pool.push_back(e);
  }
  return p.pool[p.next++];
}
void profile_record(const char* name, double bytes, cudaEvent_t begin, cudaEvent_t end) {
  profile_state().records.push_back({name, bytes, begin, end, 0.0});
}
int64_t profile_last() {
  auto& p = profile_state();
  return p.on && !p.records.empty() ? int64_t(p.records.size()) - 1 : -1;
}
void profile_add_bytes(int64_t record, double bytes) {
  auto& p = profile_state();
  if (record >= 0 && size_t(record) < p.records.size()) p.records[size_t(record)].bytes += bytes;
}
void profile_sync(const char* label, double ms) {
  profile_state().records.push_back({std::string("sync: ") + label, 0.0, nullptr, nullptr, ms});
}
void profile_enable(bool on) {
  auto& p = profile_state();
  p.on = on;
  p.records.clear();
  p.next = 0;
}
// Aggregates recorded launches by kernel name: launches, total ms, total bytes.
std::vector<ProfileSummary> profile_summary() {
  auto& p = profile_state();
  check(cudaDeviceSynchronize(), "profile sync");
  std::vector<ProfileSummary> out;
  for (const auto& r : p.records) {
    float ms = float(r.host_ms);
    if (r.begin) check(cudaEventElapsedTime(&ms, r.begin, r.end), "cudaEventElapsedTime");
    ProfileSummary* s = nullptr;
    for (auto& o : out)
      if (o.name == r.name) s = &o;
    if (!s) {
      out.push_back({r.name, 0, 0.0, 0.0});
      s = &out.back();
    }
    s->launches += 1;
    s->ms += ms;
    s->bytes += r.bytes;
  }
  return out;
}
void set_last_error(const std::string& s) { g_last_error = s; }
const char* last_error() { return g_last_error.c_str(); }

}  // namespace gpp
