// Symmetry folding: colour refinement of the rows and columns, the quotient
// ("folded") LP of the final colours, and the map back to the original.
//
// Reference: run_folding (cpp/src/folding/folding.cu:69-133), refine_color
// (folding_refinement.cu:222-359), update_color_id (folding_kernels.cu:
// 165-210), reduce_size (folding_reduce.cu:244-565), build_device_map and the
// unfold kernels (folding_map.cu:55-110, 318-380).
//
// Colours start from the row sides (AL, then AU) and the column data (c, l,
// u); every round gives each colour a pseudo-random signature (SplitMix64
// finaliser + Box-Muller, seeded by round and side), forms column signatures
// A^T sig_row and row signatures A sig_col, and splits each colour by the
// single-precision value of its members' signatures (members closer than the
// tolerance stay together).  Refinement stops when no colour splits, or gives
// up when both sides keep more than 80% distinct colours.  Sorting the
// (colour, signature) pairs uses this engine's stable radix sort on a 64-bit
// key (colour id, order-preserving float bits), so equal pairs keep index
// order as the reference's stable merge sort does.
// Folded LP: A_f[R][C] = sum over entries of colour pair (R, C) of a_ij /
// |R|, kept when |sum| > tolerance; c_f = sum of member costs; l, u, AL, AU =
// member averages (count * value when all members are equal and that product
// is exact).  The entry sums run in original entry order; colour sums in
// member index order.
#include <chrono>
#include <cmath>

#include "folding.hpp"
#include "sort.hpp"

namespace gpp {

namespace {

constexpr double kMaxReduceFraction = 0.8;
constexpr double kTwoPi = 6.283185307179586476925286766559;

__host__ __device__ __forceinline__ uint64_t splitmix_finalize(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double unit_of(uint64_t x) {
  const double u = double(splitmix_finalize(x) >> 11) * 0x1.0p-53;
  return u > 0.0 ? u : 0x1.0p-53;
}
uint64_t round_seed(int32_t round, uint64_t side) {
  return splitmix_finalize(uint64_t(round) ^ (side * 0x9e3779b97f4a7c15ULL));
}
__device__ __forceinline__ double color_signature(uint64_t seed, int32_t color) {
  const uint64_t cu = uint64_t(color);
  const double u1 = unit_of(seed ^ (cu * 0xbf58476d1ce4e5b9ULL));
  const double u2 = unit_of((seed + 0x9e3779b97f4a7c15ULL) ^ (cu * 0x94d049bb133111ebULL));
  return sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
}

// Order-preserving 32-bit image of a float (negatives reversed below positives).
__device__ __forceinline__ uint32_t float_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void fd_pack(int n, const int32_t* __restrict__ ids, const double* __restrict__ sig,
                        uint64_t* __restrict__ keys, int32_t* __restrict__ perm) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys[i] = (uint64_t(uint32_t(ids[i])) << 32) | float_key(float(sig[i]));
    perm[i] = i;
  }
}
// kernel_mark_color_start (folding_kernels.cu:75-90).
__global__ void fd_starts(int n, const uint64_t* __restrict__ keys, double tol, int32_t* __restrict__ start) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i == 0) { start[i] = 1; continue; }
    const uint64_t a = keys[i - 1], b = keys[i];
    const bool new_id = (a >> 32) != (b >> 32);
    const bool new_sig = double(key_float(uint32_t(b))) > double(key_float(uint32_t(a))) + tol;
    start[i] = new_id || new_sig ? 1 : 0;
  }
}
__global__ void fd_write(int n, const int32_t* __restrict__ perm, const int32_t* __restrict__ start,
                         const int32_t* __restrict__ excl, int write_sig, uint64_t seed, int32_t* __restrict__ ids,
                         double* __restrict__ sig_out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int id = excl[i] + start[i];   // inclusive scan: colours are 1-based
    const int member = perm[i];
    ids[member] = id;
    if (write_sig) sig_out[member] = color_signature(seed, id);
  }
}
__global__ void fd_signatures(int n, const int32_t* __restrict__ ids, uint64_t seed, double* __restrict__ sig) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    sig[i] = color_signature(seed, ids[i]);
}

// y = M x, one warp per row; lane 0 adds the row's products in stored order.
__global__ void fd_spmv(int rows, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                        const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
    double acc = 0.0;
    for (offset_t chunk = ptr[r]; chunk < ptr[r + 1]; chunk += 32) {
      const offset_t p = chunk + lane;
      const double t = p < ptr[r + 1] ? val[p] * x[idx[p]] : 0.0;
      const int live = int(min(offset_t(32), ptr[r + 1] - chunk));
      for (int k = 0; k < live; ++k) {
        const double v = __shfl_sync(0xffffffffu, t, k);
        if (lane == 0) acc += v;
      }
    }
    if (lane == 0) y[r] = acc;
  }
}

struct Side {
  int n = 0;
  int colors = 1;
  DBuf<int32_t> ids, perm, start, excl;
  DBuf<uint64_t> keys;
  DBuf<double> sig;
  void alloc(int count, cudaStream_t s) {
    n = count;
    ids.alloc(size_t(n), s);
    perm.alloc(size_t(n), s);
    start.alloc(size_t(n) + 1, s);
    excl.alloc(size_t(n) + 1, s);
    keys.alloc(size_t(n), s);
    sig.alloc(size_t(n), s);
    ids.zero();
  }
  // update_color_id (folding_kernels.cu:165-210): split colours by the float
  // value of `value`; optionally write each member's new colour signature.
  void update(const double* value, double tol, bool write_sig, uint64_t seed, cudaStream_t s) {
    const int g = grid_stride_blocks(n);
    GPP_LAUNCH(fd_pack, g, kThreads, 0, s, n, ids.p, value, keys.p, perm.p);
    radix_sort_pairs(keys.p, perm.p, n, s);
    GPP_LAUNCH(fd_starts, g, kThreads, 0, s, n, keys.p, tol, start.p);
    exclusive_scan_i32(start.p, excl.p, n, s);
    GPP_LAUNCH(fd_write, g, kThreads, 0, s, n, perm.p, start.p, excl.p, int(write_sig), seed, ids.p, sig.p);
  }
  int count() { return read_scalar(excl.p + n); }
};

bool too_little(const Side& r, const Side& c) {
  return double(r.colors) > kMaxReduceFraction * double(r.n) && double(c.colors) > kMaxReduceFraction * double(c.n);
}

// refine_color (folding_refinement.cu:222-359), the batched variant.
bool refine(const gpp_lp& lp, double tol, Side& rows, Side& cols, cudaStream_t s) {
  rows.update(lp.AL, tol, false, 0, s);
  rows.update(lp.AU, tol, false, 0, s);
  cols.update(lp.c, tol, false, 0, s);
  cols.update(lp.l, tol, false, 0, s);
  cols.update(lp.u, tol, false, 0, s);
  rows.colors = rows.count();
  cols.colors = cols.count();
  GPP_LAUNCH(fd_signatures, grid_stride_blocks(rows.n), kThreads, 0, s, rows.n, rows.ids.p, round_seed(0, 2),
             rows.sig.p);
  GPP_LAUNCH(fd_signatures, grid_stride_blocks(cols.n), kThreads, 0, s, cols.n, cols.ids.p, round_seed(0, 5),
             cols.sig.p);
  if (too_little(rows, cols)) return false;
  DBuf<double> col_value(size_t(cols.n), s), row_value(size_t(rows.n), s);
  const int max_round = std::max(1, rows.n + cols.n);
  const int gr = std::max(1, std::min((cols.n + 7) / 8, kNumSMs * 16));
  const int gc = std::max(1, std::min((rows.n + 7) / 8, kNumSMs * 16));
  for (int round = 1; round <= max_round; ++round) {
    GPP_LAUNCH(fd_spmv, gr, kThreads, 0, s, cols.n, lp.AT.rowPtr, lp.AT.colVal, lp.AT.nzVal, rows.sig.p,
               col_value.p);
    const int prev_cols = cols.colors, prev_rows = rows.colors;
    cols.update(col_value.p, tol, true, round_seed(round, 1), s);
    GPP_LAUNCH(fd_spmv, gc, kThreads, 0, s, rows.n, lp.A.rowPtr, lp.A.colVal, lp.A.nzVal, cols.sig.p, row_value.p);
    rows.update(row_value.p, tol, true, round_seed(round, 2), s);
    rows.colors = rows.count();
    cols.colors = cols.count();
    if (too_little(rows, cols)) return false;
    if (!(rows.colors > prev_rows || cols.colors > prev_cols)) return true;
  }
  return true;
}

// ---- quotient LP ----------------------------------------------------------

__global__ void fd_count(int n, const int32_t* __restrict__ ids, int32_t* __restrict__ counts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) atomicAdd(counts + ids[i] - 1, 1);
}
__global__ void fd_member_keys(int n, const int32_t* __restrict__ ids, uint64_t* __restrict__ keys,
                               int32_t* __restrict__ vals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys[i] = (uint64_t(uint32_t(ids[i] - 1)) << 32) | uint32_t(i);
    vals[i] = i;
  }
}
// kernel_check_color_constants (folding_reduce.cu:120-140): bit 1 value,
// bit 2 lower, bit 4 upper differ from the colour's first member.
__global__ void fd_nonconstant(int n, const int32_t* __restrict__ members, const int32_t* __restrict__ ids,
                               const int32_t* __restrict__ offsets, const double* __restrict__ value,
                               const double* __restrict__ lo, const double* __restrict__ hi,
                               uint32_t* __restrict__ flags) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int member = members[p];
    const int color = ids[member] - 1;
    const int first = members[offsets[color]];
    uint32_t mask = 0;
    if (value && value[member] != value[first]) mask |= 1u;
    if (lo[member] != lo[first]) mask |= 2u;
    if (hi[member] != hi[first]) mask |= 4u;
    if (mask) atomicOr(flags + color, mask);
  }
}

// True when count * value equals the left-to-right sum of count copies of
// value exactly: the value's odd significand times count stays below 2^53.
__device__ bool exact_repeat_sum(double value, int count, double& sum) {
  if (value == 0.0) { sum = 0.0; return true; }
  if (isinf(value)) { sum = value; return true; }
  if (!isfinite(value) || count <= 0) return false;
  const uint64_t bits = uint64_t(__double_as_longlong(value)) & 0x7fffffffffffffffULL;
  uint64_t mant = bits & 0xfffffffffffffULL;
  if (bits >> 52) mant |= 1ULL << 52;
  mant >>= (__ffsll((long long)mant) - 1);
  if (mant > (1ULL << 53) / uint32_t(count)) return false;
  const double product = value * double(count);
  if (!isfinite(product)) return false;
  sum = product;
  return true;
}

// kernel_reduce_color_values_constant / _bounds_constant (folding_reduce.cu:
// 163-235): sums in member order, averages for bounds and sides.
__global__ void fd_reduce_values(int colors, const int32_t* __restrict__ members, const int32_t* __restrict__ offsets,
                                 const int32_t* __restrict__ counts, const uint32_t* __restrict__ flags,
                                 const double* __restrict__ value, double* __restrict__ out) {
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < colors; col += gridDim.x * blockDim.x) {
    const int b = offsets[col], k = counts[col];
    double sum = 0.0;
    if (!(flags[col] & 1u) && exact_repeat_sum(value[members[b]], k, sum)) { out[col] = sum; continue; }
    sum = 0.0;
    for (int p = b; p < b + k; ++p) sum += value[members[p]];
    out[col] = sum;
  }
}
__global__ void fd_reduce_bounds(int colors, const int32_t* __restrict__ members, const int32_t* __restrict__ offsets,
                                 const int32_t* __restrict__ counts, const uint32_t* __restrict__ flags,
                                 const double* __restrict__ lo, const double* __restrict__ hi,
                                 double* __restrict__ lo_out, double* __restrict__ hi_out) {
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < colors; col += gridDim.x * blockDim.x) {
    const int b = offsets[col], k = counts[col];
    double ls = 0.0, us = 0.0;
    const bool le = !(flags[col] & 2u) && exact_repeat_sum(lo[members[b]], k, ls);
    const bool ue = !(flags[col] & 4u) && exact_repeat_sum(hi[members[b]], k, us);
    if (!(le && ue)) {
      if (!le) ls = 0.0;
      if (!ue) us = 0.0;
      for (int p = b; p < b + k; ++p) {
        if (!le) ls += lo[members[p]];
        if (!ue) us += hi[members[p]];
      }
    }
    lo_out[col] = ls / double(k);
    hi_out[col] = us / double(k);
  }
}

// kernel_emit_triplet_warp (folding_reduce.cu:52-74): entry key (R-1)*C +
// (C-1), value a_ij / |R|.
__global__ void fd_entries(int rows, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ val, const int32_t* __restrict__ rid,
                           const int32_t* __restrict__ cid, const int32_t* __restrict__ rcount, int ncc,
                           uint64_t* __restrict__ keys, int32_t* __restrict__ order, double* __restrict__ weighted) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
    const int R = rid[r];
    const double w = 1.0 / double(rcount[R - 1]);
    for (offset_t p = ptr[r] + lane; p < ptr[r + 1]; p += 32) {
      keys[p] = uint64_t(R - 1) * uint64_t(ncc) + uint64_t(cid[idx[p]] - 1);
      order[p] = int32_t(p);
      weighted[p] = val[p] * w;
    }
  }
}
__global__ void fd_heads(int64_t n, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
  for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n; q += int64_t(gridDim.x) * blockDim.x)
    head[q] = q == 0 || keys[q] != keys[q - 1] ? 1 : 0;
}
// One thread per distinct key: its entries summed in original entry order;
// kept when |sum| > tolerance.
__global__ void fd_sum_unique(int64_t n, const int32_t* __restrict__ head, const int32_t* __restrict__ hpos,
                              const int32_t* __restrict__ order, const double* __restrict__ weighted,
                              double tol, double* __restrict__ usum, int32_t* __restrict__ keep) {
  for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n; q += int64_t(gridDim.x) * blockDim.x) {
    if (!head[q]) continue;
    double sum = 0.0;
    int64_t e = q;
    do { sum += weighted[order[e]]; ++e; } while (e < n && !head[e]);
    usum[hpos[q]] = sum;
    keep[hpos[q]] = fabs(sum) > tol ? 1 : 0;
  }
}
__global__ void fd_write_entries(int64_t n, const int32_t* __restrict__ head, const int32_t* __restrict__ hpos,
                                 const uint64_t* __restrict__ keys, const double* __restrict__ usum,
                                 const int32_t* __restrict__ keep, const int32_t* __restrict__ kpos, int ncc,
                                 int32_t* __restrict__ row_cnt, int32_t* __restrict__ oidx, double* __restrict__ oval) {
  for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n; q += int64_t(gridDim.x) * blockDim.x) {
    if (!head[q]) continue;
    const int u = hpos[q];
    if (!keep[u]) continue;
    const int o = kpos[u];
    oidx[o] = int32_t(keys[q] % uint64_t(ncc));
    oval[o] = usum[u];
    atomicAdd(row_cnt + int(keys[q] / uint64_t(ncc)), 1);
  }
}

__global__ void fd_scale(int n, const int32_t* __restrict__ ids, const int32_t* __restrict__ counts,
                         double* __restrict__ scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    scale[i] = 1.0 / double(counts[ids[i] - 1]);
}

// kernel_unfold_cols / kernel_unfold_rows (folding_map.cu:72-110).
__global__ void fd_unfold(int n, const int32_t* __restrict__ ids, const double* __restrict__ scale,
                          const double* __restrict__ value, double* __restrict__ out, int scaled) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = scaled ? value[ids[i] - 1] * scale[i] : value[ids[i] - 1];
}

struct Members {
  DBuf<int32_t> counts, offsets, list;
  DBuf<uint32_t> flags;
};

void members_of(const Side& side, const double* value, const double* lo, const double* hi, Members& mb,
                cudaStream_t s) {
  const int n = side.n, k = side.colors;
  mb.counts.alloc(size_t(k) + 1, s);
  mb.counts.zero();
  mb.offsets.alloc(size_t(k) + 1, s);
  mb.list.alloc(size_t(n), s);
  mb.flags.alloc(size_t(k), s);
  mb.flags.zero();
  const int g = grid_stride_blocks(n);
  GPP_LAUNCH(fd_count, g, kThreads, 0, s, n, side.ids.p, mb.counts.p);
  exclusive_scan_i32(mb.counts.p, mb.offsets.p, k, s);
  DBuf<uint64_t> keys(size_t(n), s);
  GPP_LAUNCH(fd_member_keys, g, kThreads, 0, s, n, side.ids.p, keys.p, mb.list.p);
  radix_sort_pairs(keys.p, mb.list.p, n, s);
  GPP_LAUNCH(fd_nonconstant, g, kThreads, 0, s, n, mb.list.p, side.ids.p, mb.offsets.p, value, lo, hi, mb.flags.p);
}

}  // namespace

void run_folding(const gpp_lp& lp, double tolerance, FoldingResult& out) {
  if (!std::isfinite(tolerance) || tolerance < 0.0)
    throw std::invalid_argument("folding tolerance must be finite and nonnegative");
  const auto t0 = std::chrono::steady_clock::now();
  out.original_rows = out.folded_rows = lp.A.rows;
  out.original_cols = out.folded_cols = lp.A.cols;
  if (lp.A.rows == 0 || lp.A.cols == 0) return;
  auto s = ctx().stream;
  Side rows, cols;
  rows.alloc(lp.A.rows, s);
  cols.alloc(lp.A.cols, s);
  const bool ok = refine(lp, tolerance, rows, cols, s);
  if (!ok || (rows.colors == rows.n && cols.colors == cols.n)) {
    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return;
  }
  const int mr = rows.colors, nc = cols.colors;

  // reduce_size (folding_reduce.cu:244-565).
  Members rm, cm;
  members_of(rows, nullptr, lp.AL, lp.AU, rm, s);
  members_of(cols, lp.c, lp.l, lp.u, cm, s);
  const int64_t nnz = lp.A.nnz;
  DevCsr A;
  A.rows = mr;
  A.cols = nc;
  A.ptr = dalloc<offset_t>(size_t(mr) + 1);
  if (nnz > 0) {
    DBuf<uint64_t> keys(size_t(nnz), s);
    DBuf<int32_t> order(size_t(nnz), s), head(size_t(nnz) + 1, s), hpos(size_t(nnz) + 1, s);
    DBuf<double> weighted(size_t(nnz), s);
    GPP_LAUNCH(fd_entries, std::max(1, std::min((lp.A.rows + 7) / 8, kNumSMs * 16)), kThreads, 0, s, lp.A.rows,
               lp.A.rowPtr, lp.A.colVal, lp.A.nzVal, rows.ids.p, cols.ids.p, rm.counts.p, nc, keys.p, order.p,
               weighted.p);
    radix_sort_pairs(keys.p, order.p, nnz, s);
    const int g = grid_stride_blocks(nnz);
    GPP_LAUNCH(fd_heads, g, kThreads, 0, s, nnz, keys.p, head.p);
    exclusive_scan_i32(head.p, hpos.p, nnz, s);
    const int unique = read_scalar(hpos.p + nnz);
    DBuf<double> usum(size_t(unique), s);
    DBuf<int32_t> keep(size_t(unique) + 1, s), kpos(size_t(unique) + 1, s), row_cnt(size_t(mr) + 1, s);
    GPP_LAUNCH(fd_sum_unique, g, kThreads, 0, s, nnz, head.p, hpos.p, order.p, weighted.p, tolerance, usum.p, keep.p);
    exclusive_scan_i32(keep.p, kpos.p, unique, s);
    A.nnz = read_scalar(kpos.p + unique);
    A.idx = dalloc<int32_t>(size_t(A.nnz));
    A.val = dalloc<double>(size_t(A.nnz));
    row_cnt.zero();
    GPP_LAUNCH(fd_write_entries, g, kThreads, 0, s, nnz, head.p, hpos.p, keys.p, usum.p, keep.p, kpos.p, nc,
               row_cnt.p, A.idx, A.val);
    exclusive_scan_i32(row_cnt.p, A.ptr, mr, s);
  } else {
    check(cudaMemsetAsync(A.ptr, 0, sizeof(offset_t) * (size_t(mr) + 1), s), "folded empty ptr");
  }
  const DevCsr AT = transpose_csr(A, s);
  double* c = dalloc<double>(size_t(nc));
  double* l = dalloc<double>(size_t(nc));
  double* u = dalloc<double>(size_t(nc));
  double* AL = dalloc<double>(size_t(mr));
  double* AU = dalloc<double>(size_t(mr));
  GPP_LAUNCH(fd_reduce_values, grid_stride_blocks(nc), kThreads, 0, s, nc, cm.list.p, cm.offsets.p, cm.counts.p,
             cm.flags.p, lp.c, c);
  GPP_LAUNCH(fd_reduce_bounds, grid_stride_blocks(nc), kThreads, 0, s, nc, cm.list.p, cm.offsets.p, cm.counts.p,
             cm.flags.p, lp.l, lp.u, l, u);
  GPP_LAUNCH(fd_reduce_bounds, grid_stride_blocks(mr), kThreads, 0, s, mr, rm.list.p, rm.offsets.p, rm.counts.p,
             rm.flags.p, lp.AL, lp.AU, AL, AU);
  out.folded = gpp_lp{{A.rows, A.cols, A.nnz, A.ptr, A.idx, A.val},
                      {AT.rows, AT.cols, AT.nnz, AT.ptr, AT.idx, AT.val},
                      c, AL, AU, l, u, lp.obj_constant, 0, nullptr};
  // build_device_map (folding_map.cu:106-249).
  out.row_color = std::move(rows.ids);
  out.col_color = std::move(cols.ids);
  out.row_scale.alloc(size_t(rows.n), s);
  out.col_scale.alloc(size_t(cols.n), s);
  GPP_LAUNCH(fd_scale, grid_stride_blocks(rows.n), kThreads, 0, s, rows.n, out.row_color.p, rm.counts.p,
             out.row_scale.p);
  GPP_LAUNCH(fd_scale, grid_stride_blocks(cols.n), kThreads, 0, s, cols.n, out.col_color.p, cm.counts.p,
             out.col_scale.p);
  // At least one side lost colours (checked above), so the fold applies.
  out.applied = true;
  out.folded_rows = mr;
  out.folded_cols = nc;
  ctx().sync("folding");
  out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void free_folding(FoldingResult& f) {
  if (f.applied) {
    DevCsr A{f.folded.A.rows, f.folded.A.cols, f.folded.A.nnz, f.folded.A.rowPtr, f.folded.A.colVal, f.folded.A.nzVal};
    DevCsr AT{f.folded.AT.rows, f.folded.AT.cols, f.folded.AT.nnz, f.folded.AT.rowPtr, f.folded.AT.colVal,
              f.folded.AT.nzVal};
    free_csr(A);
    free_csr(AT);
    dfree(f.folded.c); dfree(f.folded.l); dfree(f.folded.u); dfree(f.folded.AL); dfree(f.folded.AU);
  }
  const int32_t r = f.original_rows, c = f.original_cols;
  f = FoldingResult{};
  f.original_rows = f.folded_rows = r;
  f.original_cols = f.folded_cols = c;
}

void unfold_to_host(const FoldingResult& f, const double* x, const double* y, const double* z, double* x_out,
                    double* y_out, double* z_out) {
  auto s = ctx().stream;
  const int n = f.original_cols, m = f.original_rows;
  DBuf<double> xo(size_t(std::max(n, 1)), s), yo(size_t(std::max(m, 1)), s), zo(size_t(std::max(n, 1)), s);
  if (x && x_out && n) {
    GPP_LAUNCH(fd_unfold, grid_stride_blocks(n), kThreads, 0, s, n, f.col_color.p, f.col_scale.p, x, xo.p, 0);
    check(cudaMemcpyAsync(x_out, xo.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "unfold x");
  }
  if (y && y_out && m) {
    GPP_LAUNCH(fd_unfold, grid_stride_blocks(m), kThreads, 0, s, m, f.row_color.p, f.row_scale.p, y, yo.p, 1);
    check(cudaMemcpyAsync(y_out, yo.p, sizeof(double) * m, cudaMemcpyDeviceToHost, s), "unfold y");
  }
  if (z && z_out && n) {
    GPP_LAUNCH(fd_unfold, grid_stride_blocks(n), kThreads, 0, s, n, f.col_color.p, f.col_scale.p, z, zo.p, 1);
    check(cudaMemcpyAsync(z_out, zo.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "unfold z");
  }
  ctx().sync("unfold");
}

}  // namespace gpp
