// Parallel rows and parallel columns: hash the pivot-normalised live pattern
// of every row (column), sort by (hash, index), then resolve each hash group
// with an exact proportionality check.
//
// Reference: rules/rule_parallel_rows.cu:132-888 and
// rules/rule_parallel_columns.cu:158-1129.  The hash is the reference's FNV-1a
// fold (sequential, or XOR-aggregated when nnz > 32 m) so that groups, and
// therefore every decision, coincide with the reference's.  The reference's
// signature pre-filter only removes rows that cannot share a full hash group
// (and its audit checks exactly that), so hashing every live row gives the
// same groups.
#include <climits>

#include "engine.cuh"
#include "folding.hpp"
#include "sort.hpp"

namespace gpp {

namespace {

constexpr uint64_t kFnvOffset = 0xcbf29ce484222325ULL;
constexpr uint64_t kFnvPrime = 0x100000001b3ULL;
__host__ __device__ __forceinline__ uint64_t mix(uint64_t h, uint64_t x) { return (h ^ x) * kFnvPrime; }
__device__ __forceinline__ uint64_t dbits(double v) { return uint64_t(__double_as_longlong(v)); }

// Row hash of one row (any schedule: the result depends only on the row).
struct RowHashArgs {
  const offset_t* ptr;
  const int32_t* idx;
  const double* val;
  const uint8_t* keep_row;
  const uint8_t* keep_col;
  double tol;
  bool use_xor;
  uint64_t* out;
};

__device__ void row_hash_thread(const RowHashArgs& g, int i) {
  if (!g.keep_row[i]) { g.out[i] = uint64_t(i); return; }
  offset_t first = -1, len = 0;
  for (offset_t p = g.ptr[i]; p < g.ptr[i + 1]; ++p)
    if (!g.keep_col || g.keep_col[g.idx[p]]) { if (first < 0) first = p; ++len; }
  if (len == 0 || fabs(g.val[first]) <= g.tol) { g.out[i] = mix(kFnvOffset, uint64_t(i)); return; }
  const double pivot = g.val[first];
  uint64_t h = mix(kFnvOffset, uint64_t(len)), agg = 0;
  for (offset_t p = first; p < g.ptr[i + 1]; ++p) {
    if (g.keep_col && !g.keep_col[g.idx[p]]) continue;
    const uint64_t b = dbits(g.val[p] / pivot);
    if (g.use_xor) agg ^= mix(mix(kFnvOffset, uint64_t(g.idx[p])), b);
    else h = mix(mix(h, uint64_t(g.idx[p])), b);
  }
  g.out[i] = g.use_xor ? mix(h, agg) : h;
}

// Warp-cooperative version for longer rows: lanes find the first live entry
// and the live length, XOR aggregates reduce across lanes, the sequential fold
// is done by lane 0 in stored order.
__device__ void row_hash_warp(const RowHashArgs& g, int i) {
  const int lane = threadIdx.x & 31;
  if (!g.keep_row[i]) { if (lane == 0) g.out[i] = uint64_t(i); return; }
  const offset_t a = g.ptr[i], e = g.ptr[i + 1];
  long long first = LLONG_MAX;
  int len = 0;
  for (offset_t p = a + lane; p < e; p += 32)
    if (!g.keep_col || g.keep_col[g.idx[p]]) { first = min(first, (long long)p); ++len; }
  for (int off = 16; off; off >>= 1) {
    len += __shfl_xor_sync(0xffffffffu, len, off);
    first = min(first, __shfl_xor_sync(0xffffffffu, first, off));
  }
  if (len == 0 || fabs(g.val[first]) <= g.tol) { if (lane == 0) g.out[i] = mix(kFnvOffset, uint64_t(i)); return; }
  const double pivot = g.val[first];
  const uint64_t h0 = mix(kFnvOffset, uint64_t(len));
  if (g.use_xor) {
    uint64_t agg = 0;
    for (offset_t p = first + lane; p < e; p += 32) {
      if (g.keep_col && !g.keep_col[g.idx[p]]) continue;
      agg ^= mix(mix(kFnvOffset, uint64_t(g.idx[p])), dbits(g.val[p] / pivot));
    }
    for (int off = 16; off; off >>= 1) agg ^= __shfl_xor_sync(0xffffffffu, agg, off);
    if (lane == 0) g.out[i] = mix(h0, agg);
  } else {
    uint64_t h = h0;
    for (offset_t chunk = first; chunk < e; chunk += 32) {
      const offset_t p = chunk + lane;
      const bool live = p < e && (!g.keep_col || g.keep_col[g.idx[p]]);
      const uint64_t col = live ? uint64_t(g.idx[p]) : 0;
      const uint64_t b = live ? dbits(g.val[p] / pivot) : 0;
      const unsigned mask = __ballot_sync(0xffffffffu, live);
      for (int t = 0; t < 32; ++t) {
        const uint64_t ct = __shfl_sync(0xffffffffu, col, t);
        const uint64_t bt = __shfl_sync(0xffffffffu, b, t);
        if ((mask >> t) & 1u) h = mix(mix(h, ct), bt);
      }
    }
    if (lane == 0) g.out[i] = h;
  }
}

// Four rows per warp, eight lanes (a group) per row, eight stored entries per
// round.  A first sweep finds the live length and the first live entry (the
// pivot); the second forms the hash: the XOR aggregate is order-free, the
// sequential fold visits the group's live entries of each round in stored
// order through shuffles.  Every lane runs the same number of rounds (the
// warp's maximum), so ballots and shuffles stay warp-uniform; rounds past a
// row's end have no live entry.
__device__ void row_hash_grouped(const RowHashArgs& g, int i) {
  const int lane = threadIdx.x & 31, group = lane >> 3, gl = lane & 7;
  const unsigned shift = unsigned(group * 8);
  const bool keep = i >= 0 && g.keep_row[i];
  const offset_t a = keep ? g.ptr[i] : 0, e = keep ? g.ptr[i + 1] : 0;
  const int rounds = __reduce_max_sync(0xffffffffu, int((e - a + 7) >> 3));
  int len = 0;
  offset_t first = -1;
  for (int k = 0; k < rounds; ++k) {
    const offset_t p = a + offset_t(k) * 8 + gl;
    const bool live = p < e && (!g.keep_col || g.keep_col[__ldcs(g.idx + p)]);
    const unsigned bits = (__ballot_sync(0xffffffffu, live) >> shift) & 0xFFu;
    if (first < 0 && bits) first = a + offset_t(k) * 8 + (__ffs(bits) - 1);
    len += __popc(bits);
  }
  const bool trivial = !keep || len == 0 || fabs(g.val[first]) <= g.tol;
  const double pivot = trivial ? 1.0 : g.val[first];
  const offset_t from = trivial ? e : first;
  const int rounds2 = __reduce_max_sync(0xffffffffu, int((e - from + 7) >> 3));
  uint64_t h = mix(kFnvOffset, uint64_t(len)), agg = 0;
  for (int k = 0; k < rounds2; ++k) {
    const offset_t p = from + offset_t(k) * 8 + gl;
    const bool live = p < e && (!g.keep_col || g.keep_col[__ldcs(g.idx + p)]);
    const uint64_t col = live ? uint64_t(__ldcs(g.idx + p)) : 0;
    const uint64_t b = live ? dbits(__ldcs(g.val + p) / pivot) : 0;
    if (g.use_xor) {
      if (live) agg ^= mix(mix(kFnvOffset, col), b);
    } else {
      const unsigned bits = (__ballot_sync(0xffffffffu, live) >> shift) & 0xFFu;
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const uint64_t ct = __shfl_sync(0xffffffffu, col, t, 8);
        const uint64_t bt = __shfl_sync(0xffffffffu, b, t, 8);
        if ((bits >> t) & 1u) h = mix(mix(h, ct), bt);
      }
    }
  }
  if (g.use_xor)
    for (int off = 4; off; off >>= 1) agg ^= __shfl_xor_sync(0xffffffffu, agg, off, 8);
  if (gl == 0 && i >= 0) {
    if (!g.keep_row[i]) g.out[i] = uint64_t(i);
    else if (trivial) g.out[i] = mix(kFnvOffset, uint64_t(i));
    else g.out[i] = g.use_xor ? mix(h, agg) : h;
  }
}

__global__ void __launch_bounds__(kThreads)
row_hash_kernel(int rows, RowHashArgs g, const int32_t* __restrict__ medium, const int32_t* __restrict__ longq,
                const int32_t* __restrict__ counts, int short_blocks) {
  const int b = blockIdx.x;
  if (b < short_blocks) {
    for (int i = b * blockDim.x + threadIdx.x; i < rows; i += short_blocks * blockDim.x)
      if (g.ptr[i + 1] - g.ptr[i] <= kShortRow) row_hash_thread(g, i);
    return;
  }
  // Medium rows four to a warp; long rows (> kLongRow stored entries) one to
  // a warp, so that no group waits through a long row's rounds.
  const int nwarps = (gridDim.x - short_blocks) * (kThreads / 32);
  const int wid = (b - short_blocks) * (kThreads / 32) + (threadIdx.x >> 5);
  const int nmedium = counts[0];
  for (int q0 = wid * 4; q0 < nmedium; q0 += nwarps * 4) {
    const int q = q0 + ((threadIdx.x & 31) >> 3);
    row_hash_grouped(g, q < nmedium ? medium[q] : -1);
  }
  for (int q = wid; q < counts[1]; q += nwarps) row_hash_warp(g, longq[q]);
}

__global__ void gather_live(int n, const int32_t* __restrict__ take, const int32_t* __restrict__ pos,
                            const uint64_t* __restrict__ hash, uint64_t* __restrict__ keys, int32_t* __restrict__ ids) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (take[i]) { keys[pos[i]] = hash[i]; ids[pos[i]] = i; }
}

// Repeated-hash filter.  Only a hash that two or more live items share can
// form a group, so only those items need sorting.  Every live item takes two
// positions in a bitmap from its mixed hash (the SplitMix64 finaliser, so the
// positions are spread whatever the row hash's low bits look like), sets them
// in `seen`, and marks a position in `twice` when it finds it already set.
// An item is a candidate when both of its positions are marked.  Items with
// equal hashes have equal positions, so every group of two or more is kept
// whole; a hash held once is kept only if both of its positions collide with
// other items (with 32 bitmap positions per item, about 0.4% of them).  The
// dropped items are groups of one, which the group kernels pass over, and the
// kept ones stay in (hash, index) order, so the groups found, their order and
// every record are those of the unfiltered sort.
__device__ __forceinline__ uint64_t mix_hash(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
__global__ void mark_hash_bits(int n, const uint8_t* __restrict__ keep, const uint64_t* __restrict__ hash,
                               uint32_t* __restrict__ seen, uint32_t* __restrict__ twice, uint64_t bit_mask) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!keep[i]) continue;
    const uint64_t z = mix_hash(hash[i]);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const uint64_t b = (k ? z >> 32 : z) & bit_mask;
      const uint32_t bit = 1u << (b & 31u);
      if (atomicOr(seen + (b >> 5), bit) & bit) atomicOr(twice + (b >> 5), bit);
    }
  }
}
__global__ void flag_repeated(int n, const uint8_t* __restrict__ keep, const uint64_t* __restrict__ hash,
                              const uint32_t* __restrict__ twice, uint64_t bit_mask, int32_t* __restrict__ flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int32_t f = 0;
    if (keep[i]) {
      const uint64_t z = mix_hash(hash[i]);
      const uint64_t b0 = z & bit_mask, b1 = (z >> 32) & bit_mask;
      f = (twice[b0 >> 5] >> (b0 & 31u) & 1u) && (twice[b1 >> 5] >> (b1 & 31u) & 1u);
    }
    flag[i] = f;
  }
}

// --- parallel rows ------------------------------------------------------------
struct LiveCursor {
  offset_t p, e;
  __device__ LiveCursor(offset_t a, offset_t b, const int32_t* idx, const uint8_t* keep) : p(a), e(b) { skip(idx, keep); }
  __device__ void skip(const int32_t* idx, const uint8_t* keep) { while (keep && p < e && !keep[idx[p]]) ++p; }
};

// _parallel_row_ratio (rule_parallel_rows.cu:346-377): a_i = ratio * a_k entrywise.
__device__ bool row_ratio(int i, int k, const offset_t* ptr, const int32_t* idx, const double* val, double tol,
                          const uint8_t* keep_col, double* out) {
  LiveCursor L(ptr[i], ptr[i + 1], idx, keep_col), R(ptr[k], ptr[k + 1], idx, keep_col);
  if (L.p == L.e && R.p == R.e) { *out = 1.0; return true; }
  double ratio = 0.0;
  bool set = false;
  for (; L.p < L.e && R.p < R.e; ++L.p, ++R.p, L.skip(idx, keep_col), R.skip(idx, keep_col)) {
    if (idx[L.p] != idx[R.p]) return false;
    const double ai = val[L.p], ak = val[R.p];
    if (!set) {
      if (fabs(ak) <= tol) return false;
      ratio = ai / ak;
      set = true;
    }
    if (fabs(ai - ratio * ak) > tol) return false;
  }
  *out = ratio;
  return set && L.p == L.e && R.p == R.e;
}

__device__ __forceinline__ void scaled_interval(double lo, double hi, double r, double* sl, double* su) {
  const double a = lo * r, b = hi * r;
  if (r >= 0.0) { *sl = a; *su = b; } else { *sl = b; *su = a; }
}

// _kernel_parallel_row_groups (rule_parallel_rows.cu:415-521): one thread per
// hash group, representative and merge order exactly as the reference.
__global__ void row_groups_kernel(int count, const uint64_t* __restrict__ sh, const int32_t* __restrict__ sr,
                                  const uint8_t* __restrict__ keep_row, const uint8_t* __restrict__ keep_col,
                                  double* AL, double* AU, const offset_t* __restrict__ ptr,
                                  const int32_t* __restrict__ idx, const double* __restrict__ val, double coeff_tol,
                                  double interval_tol, uint8_t* __restrict__ del, int32_t* __restrict__ merge_to,
                                  int32_t* __restrict__ step_out, double* __restrict__ rec_vals,
                                  int32_t* __restrict__ status) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
    const uint64_t hs = sh[s];
    if (s > 0 && sh[s - 1] == hs) continue;
    int e = s;
    while (e + 1 < count && sh[e + 1] == hs) ++e;
    if (e <= s) continue;
    int seed = -1;
    bool seed_eq = false;
    for (int a = s; a <= e; ++a) {
      const int row = sr[a];
      if (!keep_row[row]) continue;
      const bool eq = isfinite(AL[row]) && isfinite(AU[row]) && fabs(AL[row] - AU[row]) <= interval_tol;
      if (seed < 0 || (eq && !seed_eq)) { seed = row; seed_eq = eq; }
    }
    if (seed < 0) continue;
    int rep = seed;
    double rsl = AL[seed], rsu = AU[seed];
    for (int a = s; a <= e; ++a) {
      const int row = sr[a];
      if (row == seed || !keep_row[row]) continue;
      double r;
      if (!row_ratio(seed, row, ptr, idx, val, coeff_tol, keep_col, &r)) continue;
      double sl, su;
      scaled_interval(AL[row], AU[row], r, &sl, &su);
      if (rsl <= sl + interval_tol && su <= rsu + interval_tol) { rep = row; rsl = sl; rsu = su; }
    }
    double rl = AL[rep], ru = AU[rep];
    bool found = false;
    int step = 0;
    for (int a = s; a <= e; ++a) {
      const int row = sr[a];
      if (row == rep || !keep_row[row]) continue;
      double r;
      if (!row_ratio(rep, row, ptr, idx, val, coeff_tol, keep_col, &r)) continue;
      found = true;
      double sl, su;
      scaled_interval(AL[row], AU[row], r, &sl, &su);
      if (fmax(rl, sl) > fmin(ru, su) + interval_tol) { atomicMax(status, 1); return; }
      ++step;
      merge_to[row] = rep;
      step_out[row] = step;
      rec_vals[5 * int64_t(row) + 0] = r;
      rec_vals[5 * int64_t(row) + 1] = rl;
      rec_vals[5 * int64_t(row) + 2] = ru;
      rec_vals[5 * int64_t(row) + 3] = AL[row];
      rec_vals[5 * int64_t(row) + 4] = AU[row];
      rl = fmax(rl, sl);
      ru = fmin(ru, su);
      del[row] = 1;
    }
    if (found) { AL[rep] = rl; AU[rep] = ru; }
  }
}

__global__ void deleted_keys(int m, const uint8_t* __restrict__ del, const int32_t* __restrict__ step,
                             const int32_t* __restrict__ pos, uint64_t* __restrict__ keys, int32_t* __restrict__ ids,
                             uint8_t* __restrict__ keep_row) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    if (del[i]) {
      keys[pos[i]] = (uint64_t(uint32_t(step[i])) << 32) | uint32_t(i);
      ids[pos[i]] = i;
      keep_row[i] = 0;
    }
}
__global__ void pack_parallel_records(int64_t count, const int32_t* __restrict__ ids, const int32_t* __restrict__ first,
                                      const double* __restrict__ rec_vals, int type, int32_t* __restrict__ types,
                                      int64_t* __restrict__ is, int64_t* __restrict__ vs, int32_t* __restrict__ idx,
                                      double* __restrict__ val) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k <= count; k += int64_t(gridDim.x) * blockDim.x) {
    is[k] = 2 * k;
    vs[k] = 5 * k;
    if (k == count) continue;
    const int d = ids[k];
    types[k] = type;
    idx[2 * k + 0] = type == 4 ? first[d] : d;   // ParallelRow: (kept, deleted); ParallelColumn: (deleted, kept)
    idx[2 * k + 1] = type == 4 ? d : first[d];
    for (int t = 0; t < 5; ++t) val[5 * k + t] = rec_vals[5 * int64_t(d) + t];
  }
}

// --- parallel columns ---------------------------------------------------------
// _kernel_parallel_column_hashes (rule_parallel_columns.cu:189-240).
__global__ void col_hash_kernel(int n, const uint8_t* __restrict__ keep_col, const uint8_t* __restrict__ keep_row,
                                const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                const double* __restrict__ val, double tol, uint64_t* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (!keep_col[j]) { out[j] = uint64_t(j); continue; }
    int len = 0;
    double pivot = 0.0;
    bool set = false;
    for (offset_t p = ptr[j]; p < ptr[j + 1]; ++p)
      if (keep_row[idx[p]] && fabs(val[p]) > tol) { ++len; if (!set) { pivot = val[p]; set = true; } }
    if (!set || len == 0) { out[j] = mix(kFnvOffset, uint64_t(j)); continue; }
    uint64_t h = mix(kFnvOffset, uint64_t(len));
    for (offset_t p = ptr[j]; p < ptr[j + 1]; ++p)
      if (keep_row[idx[p]] && fabs(val[p]) > tol) h = mix(mix(h, uint64_t(idx[p])), dbits(val[p] / pivot));
    out[j] = h;
  }
}

__device__ __forceinline__ offset_t next_live_col_entry(offset_t p, offset_t e, const int32_t* idx, const double* val,
                                                        const uint8_t* keep_row, double zt) {
  while (p < e && !(keep_row[idx[p]] && fabs(val[p]) > zt)) ++p;
  return p;
}

// _parallel_column_ratio (rule_parallel_columns.cu:262-321): a_k = ratio * a_j
// with a per-entry relative tolerance.
__device__ bool col_ratio(int j, int k, const offset_t* ptr, const int32_t* idx, const double* val,
                          const uint8_t* keep_row, double zt, double coeff_tol, double* out) {
  offset_t pj = ptr[j], pk = ptr[k];
  const offset_t ej = ptr[j + 1], ek = ptr[k + 1];
  double ratio = 0.0;
  bool set = false;
  for (;;) {
    pj = next_live_col_entry(pj, ej, idx, val, keep_row, zt);
    pk = next_live_col_entry(pk, ek, idx, val, keep_row, zt);
    if (pj >= ej || pk >= ek) break;
    if (idx[pj] != idx[pk]) return false;
    const double aj = val[pj], ak = val[pk];
    if (!set) {
      if (fabs(aj) <= zt) return false;
      ratio = ak / aj;
      if (fabs(ratio) <= zt || !isfinite(ratio)) return false;
      set = true;
    }
    const double expected = ratio * aj;
    const double scale = fmax(fabs(ak), fabs(expected));
    if (!isfinite(expected) || fabs(ak - expected) > coeff_tol * scale) return false;
    ++pj;
    ++pk;
  }
  pj = next_live_col_entry(pj, ej, idx, val, keep_row, zt);
  pk = next_live_col_entry(pk, ek, idx, val, keep_row, zt);
  if (pj < ej || pk < ek || !set) return false;
  *out = ratio;
  return true;
}

__device__ __forceinline__ bool ratio_guarded(double r, double max_abs) {
  const double a = fabs(r);
  return isfinite(max_abs) && (max_abs < 1.0 || a > max_abs || a * max_abs < 1.0);
}

// _kernel_count_small_high_ratio_parallel_groups (rule_parallel_columns.cu:400-467).
__global__ void count_guard_groups(int count, const uint64_t* __restrict__ sh, const int32_t* __restrict__ sc,
                                   const uint8_t* __restrict__ keep_col, const uint8_t* __restrict__ keep_row,
                                   const double* __restrict__ c, const offset_t* __restrict__ ptr,
                                   const int32_t* __restrict__ idx, const double* __restrict__ val, double zt,
                                   double coeff_tol, double obj_tol, double max_abs, int max_size, int stop_after,
                                   int32_t* __restrict__ out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
    // Early exit once enough groups are counted: a plain (volatile) read, as
    // an atomic read of one address from every thread serialises them.
    if (*(volatile int32_t*)out >= stop_after) return;
    const uint64_t hs = sh[s];
    if (s > 0 && sh[s - 1] == hs) continue;
    int e = s;
    while (e + 1 < count && sh[e + 1] == hs) ++e;
    const int size = e - s + 1;
    if (size < 2 || size > max_size) continue;
    bool hit = false;
    for (int a = s; a < e && !hit; ++a) {
      const int j = sc[a];
      if (!keep_col[j]) continue;
      for (int b = a + 1; b <= e; ++b) {
        const int k = sc[b];
        if (!keep_col[k]) continue;
        double r;
        if (!col_ratio(j, k, ptr, idx, val, keep_row, zt, coeff_tol, &r)) continue;
        if (fabs(c[k] - r * c[j]) > obj_tol) continue;
        if (max_abs < 1.0 || fabs(r) > max_abs || fabs(r) * max_abs < 1.0) { hit = true; break; }
      }
    }
    if (hit) atomicAdd(out, 1);
  }
}

// _kernel_parallel_column_groups (rule_parallel_columns.cu:470-628).
__global__ void col_groups_kernel(int count, const uint64_t* __restrict__ sh, const int32_t* __restrict__ sc,
                                  const uint8_t* __restrict__ keep_col, const uint8_t* __restrict__ keep_row,
                                  const double* __restrict__ c, double* l, double* u, const offset_t* __restrict__ ptr,
                                  const int32_t* __restrict__ idx, const double* __restrict__ val, double zt,
                                  double coeff_tol, double obj_tol, double max_abs, const int32_t* __restrict__ guard,
                                  int guard_min, uint8_t* __restrict__ del, uint8_t* __restrict__ fixed,
                                  double* __restrict__ fval, int32_t* __restrict__ merge_to,
                                  double* __restrict__ rec_vals, int32_t* __restrict__ status) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
    const uint64_t hs = sh[s];
    if (s > 0 && sh[s - 1] == hs) continue;
    int e = s;
    while (e + 1 < count && sh[e + 1] == hs) ++e;
    if (e <= s) continue;
    const double active_max = guard && *guard < guard_min ? INFINITY : max_abs;
    for (int a = s; a < e; ++a) {
      const int j = sc[a];
      if (!keep_col[j] || del[j] || fixed[j]) continue;
      for (int b = a + 1; b <= e; ++b) {
        const int k = sc[b];
        if (!keep_col[k] || del[k] || fixed[k]) continue;
        double r;
        if (!col_ratio(j, k, ptr, idx, val, keep_row, zt, coeff_tol, &r)) continue;
        if (ratio_guarded(r, active_max)) continue;
        const double gap = c[k] - r * c[j];
        const double tl = l[j], tu = u[j], sl = l[k], su = u[k];
        if (fabs(gap) <= obj_tol) {
          merge_to[k] = j;
          rec_vals[5 * int64_t(k) + 0] = r;
          rec_vals[5 * int64_t(k) + 1] = sl;
          rec_vals[5 * int64_t(k) + 2] = su;
          rec_vals[5 * int64_t(k) + 3] = tl;
          rec_vals[5 * int64_t(k) + 4] = tu;
          double nl = -INFINITY, nu = INFINITY;
          if (r > 0.0) { if (isfinite(tl) && isfinite(sl)) nl = tl + r * sl; }
          else if (isfinite(tl) && isfinite(su)) nl = tl + r * su;
          if (r > 0.0) { if (isfinite(tu) && isfinite(su)) nu = tu + r * su; }
          else if (isfinite(tu) && isfinite(sl)) nu = tu + r * sl;
          l[j] = nl;
          u[j] = nu;
          del[k] = 1;
          atomicMax(status + 1, 1);
          continue;
        }
        bool k_lo = false, k_hi = false, j_lo = false, j_hi = false;
        if (gap > obj_tol) {
          if (r > 0.0) { k_lo = !isfinite(tu); j_hi = !isfinite(sl); }
          else { k_lo = !isfinite(tl); j_lo = !isfinite(sl); }
        } else {
          if (r > 0.0) { k_hi = !isfinite(tl); j_lo = !isfinite(su); }
          else { k_hi = !isfinite(tu); j_hi = !isfinite(su); }
        }
        if (k_lo) {
          if (!isfinite(sl)) { atomicMax(status, 1); return; }
          fixed[k] = 1; fval[k] = sl; atomicMax(status + 2, 1);
          continue;
        } else if (k_hi) {
          if (!isfinite(su)) { atomicMax(status, 1); return; }
          fixed[k] = 1; fval[k] = su; atomicMax(status + 2, 1);
          continue;
        }
        if (j_lo) {
          if (!isfinite(tl)) { atomicMax(status, 1); return; }
          fixed[j] = 1; fval[j] = tl; atomicMax(status + 2, 1);
          break;
        } else if (j_hi) {
          if (!isfinite(tu)) { atomicMax(status, 1); return; }
          fixed[j] = 1; fval[j] = tu; atomicMax(status + 2, 1);
          break;
        }
      }
    }
  }
}

__global__ void flag_to_int(int n, const uint8_t* __restrict__ f, int32_t* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = f[i] != 0;
}
__global__ void col_apply(int n, int m, const uint8_t* __restrict__ del, const uint8_t* __restrict__ fixed,
                          const double* __restrict__ fval, const double* __restrict__ c, const double* __restrict__ shift,
                          uint8_t* __restrict__ keep_col, double* __restrict__ l, double* __restrict__ u,
                          double* __restrict__ AL, double* __restrict__ AU, double* __restrict__ contrib) {
  const int top = n > m ? n : m;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < top; q += gridDim.x * blockDim.x) {
    if (q < n) {
      contrib[q] = 0.0;
      if (del[q] || fixed[q]) {
        keep_col[q] = 0;
        if (fixed[q]) { l[q] = fval[q]; u[q] = fval[q]; contrib[q] = c[q] * fval[q]; }
      }
    }
    if (q < m && shift) { AL[q] -= shift[q]; AU[q] -= shift[q]; }
  }
}
// FixedVariable records: (col, kept rows), (value, c, coefficients).
__global__ void fixed_sizes(int n, const uint8_t* __restrict__ fx, const offset_t* __restrict__ at_ptr,
                            const int32_t* __restrict__ at_idx, const uint8_t* __restrict__ keep_row,
                            int64_t* __restrict__ recs, int64_t* __restrict__ nz) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    int64_t c = 0;
    if (fx[j])
      for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p) c += keep_row[at_idx[p]] != 0;
    recs[j] = fx[j] ? 1 : 0;
    nz[j] = c;
  }
}
__global__ void fixed_pack(int n, const uint8_t* __restrict__ fx, const offset_t* __restrict__ at_ptr,
                           const int32_t* __restrict__ at_idx, const double* __restrict__ at_val,
                           const uint8_t* __restrict__ keep_row, const double* __restrict__ fval,
                           const double* __restrict__ c, const int64_t* __restrict__ rpos,
                           const int64_t* __restrict__ npos, int32_t* __restrict__ types, int64_t* __restrict__ is,
                           int64_t* __restrict__ vs, int32_t* __restrict__ idx, double* __restrict__ val) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (j == 0) { is[0] = 0; vs[0] = 0; }
    if (!fx[j]) continue;
    const int64_t k = rpos[j], base = npos[j];
    int64_t ip = k + base, vp = 2 * k + base;
    types[k] = 0;
    idx[ip++] = j;
    val[vp++] = fval[j];
    val[vp++] = c[j];
    for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p)
      if (keep_row[at_idx[p]]) { idx[ip++] = at_idx[p]; val[vp++] = at_val[p]; }
    is[k + 1] = ip;
    vs[k + 1] = vp;
  }
}

// Sorted (hash, index) pairs of the live rows (columns) whose hash may be
// shared: all live items up to kRepeatFilterMin, past it the candidates of
// the repeated-hash filter.
constexpr int32_t kRepeatFilterMin = 32768;
int32_t sorted_live_hashes(const uint64_t* hash, const uint8_t* keep, int32_t n, DBuf<uint64_t>& keys,
                           DBuf<int32_t>& ids, cudaStream_t s) {
  DBuf<int32_t> flag(size_t(n) + 1, s), pos(size_t(n) + 1, s);
  if (n > kRepeatFilterMin) {
    // 32 bitmap positions per item, a power of two between 2^20 and 2^29.
    int lg = 20;
    while (lg < 29 && (int64_t(1) << lg) < 32 * int64_t(n)) ++lg;
    const size_t words = size_t(1) << (lg - 5);
    DBuf<uint32_t> bits(2 * words, s);
    bits.zero();
    const uint64_t bit_mask = (uint64_t(1) << lg) - 1;
    GPP_LAUNCH(mark_hash_bits, grid_stride_blocks(n), kThreads, 0, s, n, keep, hash, bits.p, bits.p + words,
               bit_mask);
    GPP_LAUNCH(flag_repeated, grid_stride_blocks(n), kThreads, 0, s, n, keep, hash, bits.p + words, bit_mask,
               flag.p);
  } else {
    GPP_LAUNCH(flag_to_int, grid_stride_blocks(n), kThreads, 0, s, n, keep, flag.p);
  }
  exclusive_scan_i32(flag.p, pos.p, n, s);
  const int32_t count = read_scalar(pos.p + n);
  keys.alloc(size_t(std::max(count, 1)), s);
  ids.alloc(size_t(std::max(count, 1)), s);
  GPP_LAUNCH(gather_live, grid_stride_blocks(n), kThreads, 0, s, n, flag.p, pos.p, hash, keys.p, ids.p);
  radix_sort_pairs(keys.p, ids.p, count, s);
  return count;
}

}  // namespace

void parallel_row_hashes(const DevCsr& A, const uint8_t* keep_row, const uint8_t* keep_col, int mode,
                         uint64_t* hashes, cudaStream_t s) {
  // compute_parallel_row_hashes (rule_parallel_rows.cu:583-627); mode < 0
  // picks XOR aggregation when nnz > 32 m.
  if (A.rows <= 0) return;
  const bool use_xor = mode >= 0 ? mode != 0 : int64_t(A.nnz) > 32LL * A.rows;
  DBuf<uint8_t> ones;
  if (!keep_row) {
    ones.alloc(size_t(A.rows), s);
    check(cudaMemsetAsync(ones.p, 1, size_t(A.rows), s), "keep all rows");
    keep_row = ones.p;
  }
  const RowSchedule& sch = stored_schedule(A);
  const int sb = grid_stride_blocks(A.rows, kThreads, 16), wb = std::min<int>(kNumSMs * 8, (A.rows + 7) / 8);
  RowHashArgs g{A.ptr, A.idx, A.val, keep_row, keep_col, 1e-10, use_xor, hashes};
  const double bytes = 4.0 * (A.rows + 1) + 12.0 * A.nnz + A.rows + (keep_col ? A.cols : 0) + 8.0 * A.rows;
  GPP_LAUNCH_BYTES(row_hash_kernel, bytes, sb + wb, kThreads, 0, s, A.rows, g, sch.medium.p, sch.long_rows.p,
                   sch.counts.p, sb);
}

void rule_parallel_rows(Plan& plan, const WorkingLp& lp, const Stats&, const gpp_params& p) {
  // apply_rule_parallel_rows (rule_parallel_rows.cu:643-888).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m();
  if (m <= 1) return;
  auto s = ctx().stream;
  DBuf<uint64_t> hash(size_t(m), s);
  {
    const bool use_xor = int64_t(lp.A.nnz) > 32LL * m;
    const RowSchedule& sch = stored_schedule(lp.A);
    const int sb = grid_stride_blocks(m, kThreads, 16), wb = std::min<int>(kNumSMs * 8, (m + 7) / 8);
    RowHashArgs g{lp.A.ptr, lp.A.idx, lp.A.val, plan.keep_row.p, plan.keep_col.p, p.zero_tol, use_xor, hash.p};
    const double bytes = 4.0 * (m + 1) + 12.0 * lp.A.nnz + m + lp.n() + 8.0 * m;
    GPP_LAUNCH_BYTES(row_hash_kernel, bytes, sb + wb, kThreads, 0, s, m, g, sch.medium.p, sch.long_rows.p,
                     sch.counts.p, sb);
  }
  DBuf<uint64_t> keys;
  DBuf<int32_t> ids;
  const int32_t count = sorted_live_hashes(hash.p, plan.keep_row.p, m, keys, ids, s);
  if (count <= 1) return;
  DBuf<uint8_t> del(size_t(m), s);
  DBuf<int32_t> merge_to(size_t(m), s), step(size_t(m), s);
  DBuf<double> rec(size_t(5) * size_t(m), s);
  del.zero();
  Status st;
  st.clear(2);
  GPP_LAUNCH(row_groups_kernel, grid_stride_blocks(count), kThreads, 0, s, count, keys.p, ids.p, plan.keep_row.p,
             plan.keep_col.p, plan.AL.p, plan.AU.p, lp.A.ptr, lp.A.idx, lp.A.val, p.zero_tol, p.feasibility_tol,
             del.p, merge_to.p, step.p, rec.p, st.d);
  if (st.read(1)[0]) { plan.has_infeasible = true; return; }
  DBuf<int32_t> flag(size_t(m) + 1, s), pos(size_t(m) + 1, s);
  GPP_LAUNCH(flag_to_int, grid_stride_blocks(m), kThreads, 0, s, m, del.p, flag.p);
  exclusive_scan_i32(flag.p, pos.p, m, s);
  const int32_t deleted = read_scalar(pos.p + m);
  if (!deleted) return;
  DBuf<uint64_t> dkeys(size_t(deleted), s);
  DBuf<int32_t> dids(size_t(deleted), s);
  GPP_LAUNCH(deleted_keys, grid_stride_blocks(m), kThreads, 0, s, m, del.p, step.p, pos.p, dkeys.p, dids.p,
             plan.keep_row.p);
  if (p.record_postsolve_tape) {
    // Records ordered by (merge step, deleted row) (rule_parallel_rows.cu:79-84).
    radix_sort_pairs(dkeys.p, dids.p, deleted, s);
    PostsolveSegment seg = make_segment(deleted, 2 * int64_t(deleted), 5 * int64_t(deleted));
    GPP_LAUNCH(pack_parallel_records, grid_stride_blocks(deleted + 1), kThreads, 0, s, int64_t(deleted), dids.p,
               merge_to.p, rec.p, 4, seg.types.p, seg.is.p, seg.vs.p, seg.idx.p, seg.val.p);
    plan.tape.push_back(std::move(seg));
  }
  plan.has_row_action = plan.has_change = true;
}

void rule_parallel_columns(Plan& plan, const WorkingLp& lp, const Stats&, const gpp_params& p) {
  // apply_rule_parallel_columns (rule_parallel_columns.cu:725-1127).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (n <= 1) return;
  auto s = ctx().stream;
  DBuf<uint64_t> hash(size_t(n), s);
  GPP_LAUNCH_BYTES(col_hash_kernel, 4.0 * (n + 1) + 12.0 * lp.AT.nnz + n + m + 8.0 * n, grid_stride_blocks(n),
                   kThreads, 0, s, n, plan.keep_col.p, plan.keep_row.p, lp.AT.ptr, lp.AT.idx, lp.AT.val, p.zero_tol,
                   hash.p);
  DBuf<uint64_t> keys;
  DBuf<int32_t> ids;
  const int32_t count = sorted_live_hashes(hash.p, plan.keep_col.p, n, keys, ids, s);
  if (count <= 1) return;
  const double coeff_tol = std::fmax(p.zero_tol, p.bound_tol), obj_tol = coeff_tol;
  const bool guard = std::isfinite(p.parallel_columns_max_abs_ratio) && p.parallel_columns_scale_guard_min_groups > 1;
  Status st;
  st.clear(4);
  if (guard)
    GPP_LAUNCH(count_guard_groups, grid_stride_blocks(count), kThreads, 0, s, count, keys.p, ids.p, plan.keep_col.p,
               plan.keep_row.p, plan.c.p, lp.AT.ptr, lp.AT.idx, lp.AT.val, p.zero_tol, coeff_tol, obj_tol,
               p.parallel_columns_max_abs_ratio, p.parallel_columns_scale_guard_max_group_size,
               p.parallel_columns_scale_guard_min_groups, st.d + 3);
  DBuf<uint8_t> del(size_t(n), s), fixed(size_t(n), s);
  DBuf<double> fval(size_t(n), s), rec(size_t(5) * size_t(n), s), contrib(size_t(n), s);
  DBuf<int32_t> merge_to(size_t(n), s);
  del.zero();
  fixed.zero();
  GPP_LAUNCH(col_groups_kernel, grid_stride_blocks(count), kThreads, 0, s, count, keys.p, ids.p, plan.keep_col.p,
             plan.keep_row.p, plan.c.p, plan.l.p, plan.u.p, lp.AT.ptr, lp.AT.idx, lp.AT.val, p.zero_tol, coeff_tol,
             obj_tol, p.parallel_columns_max_abs_ratio, guard ? st.d + 3 : nullptr,
             p.parallel_columns_scale_guard_min_groups, del.p, fixed.p, fval.p, merge_to.p, rec.p, st.d);
  const int32_t* f = st.read(3);
  if (f[0]) { plan.has_unbounded = true; return; }
  const bool merged = f[1] != 0, any_fixed = f[2] != 0;
  if (!merged && !any_fixed) return;
  if (merged && p.record_postsolve_tape) {
    // Records ordered by deleted column (rule_parallel_columns.cu:83-87).
    DBuf<int32_t> flag(size_t(n) + 1, s), pos(size_t(n) + 1, s);
    GPP_LAUNCH(flag_to_int, grid_stride_blocks(n), kThreads, 0, s, n, del.p, flag.p);
    exclusive_scan_i32(flag.p, pos.p, n, s);
    const int32_t merges = read_scalar(pos.p + n);
    DBuf<uint64_t> dkeys(size_t(merges), s);
    DBuf<int32_t> dids(size_t(merges), s);
    DBuf<uint8_t> untouched(size_t(n), s);
    untouched.copy_from(plan.keep_col.p, size_t(n));
    GPP_LAUNCH(deleted_keys, grid_stride_blocks(n), kThreads, 0, s, n, del.p, merge_to.p, pos.p, dkeys.p, dids.p,
               untouched.p);  // ids are already in ascending column order
    PostsolveSegment seg = make_segment(merges, 2 * int64_t(merges), 5 * int64_t(merges));
    GPP_LAUNCH(pack_parallel_records, grid_stride_blocks(merges + 1), kThreads, 0, s, int64_t(merges), dids.p,
               merge_to.p, rec.p, 3, seg.types.p, seg.is.p, seg.vs.p, seg.idx.p, seg.val.p);
    plan.tape.push_back(std::move(seg));
  }
  DBuf<double> shift;
  if (any_fixed) {
    if (p.record_postsolve_tape) {
      DBuf<int64_t> rc(size_t(n) + 1, s), nz(size_t(n) + 1, s), rpos(size_t(n) + 1, s), npos(size_t(n) + 1, s);
      GPP_LAUNCH(fixed_sizes, grid_stride_blocks(n), kThreads, 0, s, n, fixed.p, lp.AT.ptr, lp.AT.idx, plan.keep_row.p,
                 rc.p, nz.p);
      exclusive_scan_i64(rc.p, rpos.p, n, s);
      exclusive_scan_i64(nz.p, npos.p, n, s);
      const auto [recs, nnz] = read_scalars(rpos.p + n, npos.p + n);
      PostsolveSegment seg = make_segment(recs, recs + nnz, 2 * recs + nnz);
      GPP_LAUNCH(fixed_pack, grid_stride_blocks(n), kThreads, 0, s, n, fixed.p, lp.AT.ptr, lp.AT.idx, lp.AT.val,
                 plan.keep_row.p, fval.p, plan.c.p, rpos.p, npos.p, seg.types.p, seg.is.p, seg.vs.p, seg.idx.p,
                 seg.val.p);
      plan.tape.push_back(std::move(seg));
    }
    shift.alloc(size_t(std::max(m, 1)), s);
    if (m) row_gather_shift(lp.A, lp.AT, plan.keep_row.p, fixed.p, fval.p, nullptr, shift.p, s);
    plan.has_row_action = true;
  }
  GPP_LAUNCH(col_apply, grid_stride_blocks(std::max(n, m)), kThreads, 0, s, n, m, del.p, fixed.p, fval.p, plan.c.p,
             any_fixed ? shift.p : nullptr, plan.keep_col.p, plan.l.p, plan.u.p, plan.AL.p, plan.AU.p, contrib.p);
  plan.obj_delta += any_fixed ? det_sum(contrib.p, n, s) : 0.0;
  plan.has_col_action = plan.has_change = true;
}

}  // namespace gpp
