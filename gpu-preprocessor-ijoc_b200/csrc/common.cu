// Engine context, status block, scans and the canonical deterministic sum.
#include "common.cuh"

#include <algorithm>
#include <memory>
#include <mutex>

namespace gpp {

uint64_t& launch_counter() {
  static thread_local uint64_t count = 0;
  return count;
}

Context::Context() {
  check(cudaGetDevice(&device), "cudaGetDevice");
  // Blocking stream: implicitly ordered after work the caller queued on the
  // legacy default stream, as the reference's synchronous API assumes.
  check(cudaStreamCreateWithFlags(&stream, cudaStreamDefault), "cudaStreamCreate");
  cudaMemPool_t pool;
  check(cudaDeviceGetDefaultMemPool(&pool, device), "cudaDeviceGetDefaultMemPool");
  uint64_t keep = UINT64_MAX;  // keep freed blocks in the pool between presolve calls
  check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool threshold");
  check(cudaMallocHost(reinterpret_cast<void**>(&host_status), sizeof(int32_t) * kStatusWords),
        "cudaMallocHost status");
}

Context::~Context() {
  if (host_status) cudaFreeHost(host_status);
  if (stream) cudaStreamDestroy(stream);
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

Status::Status() { check(cudaMallocAsync(reinterpret_cast<void**>(&d), sizeof(int32_t) * Context::kStatusWords, ctx().stream), "status alloc"); }
Status::~Status() { if (d) cudaFreeAsync(d, ctx().stream); }
void Status::clear(int words) {
  check(cudaMemsetAsync(d, 0, sizeof(int32_t) * size_t(words), ctx().stream), "status clear");
}
const int32_t* Status::read(int words) {
  auto& c = ctx();
  check(cudaMemcpyAsync(c.host_status, d, sizeof(int32_t) * size_t(words), cudaMemcpyDeviceToHost, c.stream),
        "status read");
  c.sync("status sync");
  return c.host_status;
}

namespace {
constexpr int kScanTile = 2048;  // 256 threads x 8 items

template <class T>
__global__ void tile_reduce(const T* __restrict__ in, int64_t n, T* __restrict__ tile_sums) {
  __shared__ T sm[kThreads];
  const int64_t base = int64_t(blockIdx.x) * kScanTile;
  T acc = 0;
  for (int k = 0; k < kScanTile / kThreads; ++k) {
    const int64_t i = base + int64_t(k) * kThreads + threadIdx.x;
    if (i < n) acc += in[i];
  }
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sm[threadIdx.x] += sm[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = sm[0];
}

// Exclusive scan of tile sums in one block of 1024 threads.
template <class T>
__global__ void scan_tile_sums(T* sums, int64_t count, T* total_out) {
  __shared__ T sm[1024];
  const int64_t per = (count + 1023) / 1024;
  const int64_t b = int64_t(threadIdx.x) * per;
  T local = 0;
  for (int64_t k = 0; k < per && b + k < count; ++k) local += sums[b + k];
  sm[threadIdx.x] = local;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const T v = threadIdx.x >= unsigned(off) ? sm[threadIdx.x - off] : T(0);
    __syncthreads();
    sm[threadIdx.x] += v;
    __syncthreads();
  }
  T run = threadIdx.x ? sm[threadIdx.x - 1] : T(0);
  for (int64_t k = 0; k < per && b + k < count; ++k) {
    const T v = sums[b + k];
    sums[b + k] = run;
    run += v;
  }
  if (threadIdx.x == 1023) *total_out = sm[1023];
}

// Each block rescans its tile: thread t owns 8 consecutive items.
template <class T>
__global__ void tile_scan(const T* __restrict__ in, int64_t n, const T* __restrict__ tile_offsets,
                          T* __restrict__ out) {
  __shared__ T sm[kThreads];
  const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * 8;
  T v[8];
  T local = 0;
  for (int k = 0; k < 8; ++k) {
    v[k] = base + k < n ? in[base + k] : T(0);
    local += v[k];
  }
  sm[threadIdx.x] = local;
  __syncthreads();
  for (int off = 1; off < kThreads; off <<= 1) {
    const T t = threadIdx.x >= unsigned(off) ? sm[threadIdx.x - off] : T(0);
    __syncthreads();
    sm[threadIdx.x] += t;
    __syncthreads();
  }
  T run = tile_offsets[blockIdx.x] + (threadIdx.x ? sm[threadIdx.x - 1] : T(0));
  for (int k = 0; k < 8; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

template <class T>
__global__ void write_total(T* out, int64_t n, const T* total) { out[n] = *total; }

template <class T>
void exclusive_scan(const T* in, T* out, int64_t n, cudaStream_t s) {
  if (n <= 0) {
    check(cudaMemsetAsync(out, 0, sizeof(T), s), "scan empty");
    return;
  }
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  DBuf<T> sums(size_t(tiles) + 1, s);
  GPP_LAUNCH(tile_reduce<T>, int(tiles), kThreads, 0, s, in, n, sums.p);
  GPP_LAUNCH(scan_tile_sums<T>, 1, 1024, 0, s, sums.p, tiles, sums.p + tiles);
  // tile_scan reads in[] before out[] is written only within the same tile;
  // `in` and `out` may alias.
  GPP_LAUNCH(tile_scan<T>, int(tiles), kThreads, 0, s, in, n, sums.p, out);
  GPP_LAUNCH(write_total<T>, 1, 1, 0, s, out, n, sums.p + tiles);
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
  const char* name;
  double bytes;
  cudaEvent_t begin, end;
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
  profile_state().records.push_back({name, bytes, begin, end});
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
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, r.begin, r.end), "cudaEventElapsedTime");
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
