// Singleton-column rule: substitute out columns that appear in one live row.
//
// Reference: apply_rule_singleton_columns (cpp/src/presolve/rules/
// rule_singleton_columns.cu:1562-1827) with its kernels :459-1560.  The
// decisions are the reference's, evaluated against the unmodified plan:
//   * an activity cache per row holding a candidate (rows of live length
//     <= 1024 sum in stored order; longer rows give live rank k to thread
//     k mod 256 and reduce with a halving tree, :555-754);
//   * implied-free tests and the action choice (:756-903);
//   * one owner per row by atomicMin over keys that rank free eliminations
//     first, then the smallest column (:905-1018);
//   * staging (:1021-1073), the cost update c_k -= c_j a_ik / a_ij summed per
//     column in stored (row) order (:1075-1139), substitution and row-dual-
//     shift records in ascending row order (:459-508, :1191-1560).
// B200 layout of the work: the rule touches only the candidate columns, the
// rows that hold them and the columns of eliminated rows, through compacted
// work lists, instead of sweeping all of A / AT as the reference does.  The
// objective delta is the reference's canonical sum over the rule's entry
// domain, evaluated from the sparse contributions (det_sum_sparse).
#include <algorithm>
#include <climits>

#include "engine.cuh"
#include "live_visit.cuh"
#include "sort.hpp"

namespace gpp {

namespace {

enum : uint8_t {
  kNone = 0, kSetRowSide = 1, kTightenLhs = 2, kTightenRhs = 3,
  kEliminateFree = 4, kEliminateFreeAbove = 5, kEliminateFreeBelow = 6
};
// Row kinds after staging (only rows in the winner list carry one).
enum : uint8_t { kRowElimKept = 1, kRowElimDeleted = 2, kRowDualShift = 3 };

constexpr int kUnclaimed = INT_MAX;
constexpr int kClaimed = INT_MAX - 1;   // row holds a candidate, no owner yet

// Status words.
enum { kStUnbounded = 0, kStCand = 1, kStRows = 2, kStLong = 3, kStWin = 4, kStElim = 5, kStSide = 6,
       kStTouched = 7, kStWords = 8 };

__device__ __forceinline__ bool direct_unbounded(double cj, double a, double lhs, double rhs, double lb, double ub,
                                                 double zt) {
  // _singleton_column_direct_unbounded (rule_singleton_columns.cu:516-527).
  return (cj > zt && a > zt && !isfinite(lhs) && !isfinite(lb)) ||
         (cj > zt && a < -zt && !isfinite(rhs) && !isfinite(lb)) ||
         (cj < -zt && a < -zt && !isfinite(lhs) && !isfinite(ub)) ||
         (cj < -zt && a > zt && !isfinite(rhs) && !isfinite(ub));
}

// Candidates (:905-940): kept singleton column in a kept row with another
// live entry and |a| > zero_tol.  Directly unbounded candidates only raise the
// flag.  The first candidate of a row claims it for the cache and stage lists.
__global__ void sc_candidates(int n, int m, const uint8_t* __restrict__ keep_col, const uint8_t* __restrict__ keep_row,
                              const uint8_t* __restrict__ singleton, const int32_t* __restrict__ srow,
                              const double* __restrict__ sval, const int32_t* __restrict__ row_nnz,
                              const double* __restrict__ c, const double* __restrict__ l, const double* __restrict__ u,
                              const double* __restrict__ AL, const double* __restrict__ AU, double zero_tol,
                              int32_t* __restrict__ owner, int32_t* __restrict__ cand, int32_t* __restrict__ rows,
                              int32_t* __restrict__ long_rows, int32_t* st) {
  const int stride = gridDim.x * blockDim.x;
  const int top = (n + stride - 1) / stride * stride;   // every thread of a block runs the same trips
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < top; j += stride) {
    bool take = false, claim = false, is_long = false;
    if (j < n && keep_col[j] && singleton[j]) {
      const int row = srow[j];
      const double a = sval[j];
      if (row >= 0 && row < m && keep_row[row] && !(fabs(a) <= zero_tol) && row_nnz[row] > 1) {
        if (direct_unbounded(c[j], a, AL[row], AU[row], l[j], u[j], zero_tol)) {
          atomicOr(st + kStUnbounded, 1);
        } else {
          take = true;
          claim = atomicCAS(owner + row, kUnclaimed, kClaimed) == kUnclaimed;
          is_long = claim && row_nnz[row] > kLongRow;
        }
      }
    }
    const int pc = block_append(st + kStCand, take);
    if (take) cand[pc] = j;
    const int pr = block_append(st + kStRows, claim);
    if (claim) rows[pr] = srow[j];
    const int pl = block_append(st + kStLong, is_long);
    if (is_long) long_rows[pl] = srow[j];
  }
}

struct RowCache {
  double fmin, fmax;
  int min_neg, min_pos, max_neg, max_pos;
  int invalid;
};

__device__ __forceinline__ void cache_term(RowCache& r, double a, double lj, double uj) {
  const double tmin = a >= 0.0 ? a * lj : a * uj;
  const double tmax = a >= 0.0 ? a * uj : a * lj;
  if (isnan(tmin) || isnan(tmax)) { r.invalid = 1; return; }
  if (isinf(tmin)) { if (tmin < 0.0) ++r.min_neg; else ++r.min_pos; } else { r.fmin += tmin; }
  if (isinf(tmax)) { if (tmax < 0.0) ++r.max_neg; else ++r.max_pos; } else { r.fmax += tmax; }
}

struct CacheOut {
  double *fmin, *fmax;
  int4* counts;
  uint8_t* invalid;
  __device__ void store(int row, const RowCache& r) const {
    fmin[row] = r.fmin;
    fmax[row] = r.fmax;
    counts[row] = make_int4(r.min_neg, r.min_pos, r.max_neg, r.max_pos);
    invalid[row] = uint8_t(r.invalid);
  }
};

// _kernel_singleton_row_activity_cache (:555-614) for rows of live length
// <= 1024.  The reference's sequential loop skips a NaN term entirely, counts
// an infinite term and adds a finite one; the counts and the NaN flag are
// order-free, so they come from ballots, and the finite sums are formed in
// stored order by the same shuffle-add chain on every lane of the row.  A
// skipped term enters the chain as +0.0, which is exact: a sum that starts at
// +0.0 never becomes -0.0 in round-to-nearest, and x + (+0.0) == x for every
// other x.  Rows of at most 32 stored entries (nearly all) take eight lanes
// each, four rows per warp, with all of a row's loads issued before its
// chain; longer rows take a whole warp, 32 entries at a time.
__global__ void sc_cache_rows(const int32_t* __restrict__ rows, const int32_t* __restrict__ st,
                              const int32_t* __restrict__ row_nnz, const offset_t* __restrict__ ptr,
                              const int32_t* __restrict__ idx, const double* __restrict__ val,
                              const uint8_t* __restrict__ keep_col, const double* __restrict__ l,
                              const double* __restrict__ u, CacheOut out) {
  const int count = st[kStRows];
  const int lane = threadIdx.x & 31, grp = lane >> 3, gl = lane & 7;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const auto group_bits = [&](bool v) { return (__ballot_sync(0xffffffffu, v) >> (grp * 8)) & 0xffu; };
  const auto whole_row = [&](int row) {
    RowCache r{0.0, 0.0, 0, 0, 0, 0, 0};
    const offset_t end = ptr[row + 1];
    for (offset_t chunk = ptr[row]; chunk < end; chunk += 32) {
      const offset_t p = chunk + lane;
      double tmin = 0.0, tmax = 0.0;
      bool live = false;
      if (p < end) {
        const int col = __ldcs(idx + p);
        if (keep_col[col]) {
          live = true;
          const double a = __ldcs(val + p);
          tmin = a >= 0.0 ? a * l[col] : a * u[col];
          tmax = a >= 0.0 ? a * u[col] : a * l[col];
        }
      }
      const bool nan = live && (isnan(tmin) || isnan(tmax));
      const bool counted = live && !nan;
      r.invalid |= __any_sync(0xffffffffu, nan);
      r.min_neg += __popc(__ballot_sync(0xffffffffu, counted && isinf(tmin) && tmin < 0.0));
      r.min_pos += __popc(__ballot_sync(0xffffffffu, counted && isinf(tmin) && tmin > 0.0));
      r.max_neg += __popc(__ballot_sync(0xffffffffu, counted && isinf(tmax) && tmax < 0.0));
      r.max_pos += __popc(__ballot_sync(0xffffffffu, counted && isinf(tmax) && tmax > 0.0));
      const double fmin_term = counted && isfinite(tmin) ? tmin : 0.0;
      const double fmax_term = counted && isfinite(tmax) ? tmax : 0.0;
      const int n = int(min(offset_t(32), end - chunk));
      for (int k = 0; k < n; ++k) {
        r.fmin += __shfl_sync(0xffffffffu, fmin_term, k);
        r.fmax += __shfl_sync(0xffffffffu, fmax_term, k);
      }
    }
    if (lane == 0) out.store(row, r);
  };
  // Row ids two iterations ahead and row pointers and lengths one ahead, so
  // an iteration's critical path starts at its entries.
  const int step = warps * 4;
  const int w_first = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 4 + grp;
  int row_next = w_first < count ? rows[w_first] : 0;
  int row_after = w_first + step < count ? rows[w_first + step] : 0;
  int len_next = w_first < count ? row_nnz[row_next] : 0;
  offset_t first_next = w_first < count ? ptr[row_next] : 0, end_next = w_first < count ? ptr[row_next + 1] : 0;
  for (int w0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 4; w0 < count; w0 += step) {
    const int w = w0 + grp;
    const int row = row_next;
    const bool take = w < count && len_next <= kLongRow;
    const offset_t first = take ? first_next : 0, end = take ? end_next : 0;
    row_next = row_after;
    const bool more = w + step < count;
    len_next = more ? row_nnz[row_next] : 0;
    first_next = more ? ptr[row_next] : 0;
    end_next = more ? ptr[row_next + 1] : 0;
    row_after = w + 2 * step < count ? rows[w + 2 * step] : 0;
    const bool grouped = take && end - first <= 32;
    const offset_t stop = grouped ? end : first;
    int col[4];
    double a[4], lj[4], uj[4];
    bool live[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const offset_t p = first + gl + 8 * j;
      col[j] = p < stop ? __ldcs(idx + p) : -1;
      a[j] = p < stop ? __ldcs(val + p) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) live[j] = col[j] >= 0 && keep_col[col[j]];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      lj[j] = live[j] ? l[col[j]] : 0.0;
      uj[j] = live[j] ? u[col[j]] : 0.0;
    }
    RowCache r{0.0, 0.0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const double tmin = live[j] ? (a[j] >= 0.0 ? a[j] * lj[j] : a[j] * uj[j]) : 0.0;
      const double tmax = live[j] ? (a[j] >= 0.0 ? a[j] * uj[j] : a[j] * lj[j]) : 0.0;
      const bool nan = live[j] && (isnan(tmin) || isnan(tmax));
      const bool counted = live[j] && !nan;
      r.invalid |= group_bits(nan) != 0;
      r.min_neg += __popc(group_bits(counted && isinf(tmin) && tmin < 0.0));
      r.min_pos += __popc(group_bits(counted && isinf(tmin) && tmin > 0.0));
      r.max_neg += __popc(group_bits(counted && isinf(tmax) && tmax < 0.0));
      r.max_pos += __popc(group_bits(counted && isinf(tmax) && tmax > 0.0));
      const double fmin_term = counted && isfinite(tmin) ? tmin : 0.0;
      const double fmax_term = counted && isfinite(tmax) ? tmax : 0.0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        r.fmin += __shfl_sync(0xffffffffu, fmin_term, k, 8);
        r.fmax += __shfl_sync(0xffffffffu, fmax_term, k, 8);
      }
    }
    if (grouped && gl == 0) out.store(row, r);
    unsigned rest = __ballot_sync(0xffffffffu, take && !grouped && gl == 0);
    while (rest) {
      const int src = __ffs(rest) - 1;
      rest &= rest - 1;
      whole_row(__shfl_sync(0xffffffffu, row, src));
    }
  }
}

// _kernel_singleton_long_row_activity_cache (:642-754): block per row; live
// rank k goes to thread k mod 256, then a shared-memory halving tree.
__global__ void __launch_bounds__(kThreads) sc_cache_long(const int32_t* __restrict__ long_rows,
                                                          const int32_t* __restrict__ st,
                                                          const int32_t* __restrict__ row_nnz,
                                                          const offset_t* __restrict__ ptr,
                                                          const int32_t* __restrict__ idx,
                                                          const double* __restrict__ val,
                                                          const uint8_t* __restrict__ keep_col,
                                                          const double* __restrict__ l, const double* __restrict__ u,
                                                          CacheOut out) {
  __shared__ int slots[kThreads];
  __shared__ int warp_counts[8];
  __shared__ double s_min[kThreads], s_max[kThreads];
  __shared__ int s_cnt[5][kThreads];
  const int count = st[kStLong];
  const int t = threadIdx.x;
  for (int q = blockIdx.x; q < count; q += gridDim.x) {
    const int row = long_rows[q];
    const offset_t first = ptr[row], last = ptr[row + 1];
    const uint8_t* mask = row_nnz[row] != int(last - first) ? keep_col : nullptr;
    RowCache r{0.0, 0.0, 0, 0, 0, 0, 0};
    live_visit<kThreads>(first, last, idx, mask, slots, warp_counts, [&](offset_t p) {
      const int col = idx[p];
      if (keep_col[col]) cache_term(r, val[p], l[col], u[col]);
    });
    s_min[t] = r.fmin;
    s_max[t] = r.fmax;
    s_cnt[0][t] = r.min_neg; s_cnt[1][t] = r.min_pos; s_cnt[2][t] = r.max_neg; s_cnt[3][t] = r.max_pos;
    s_cnt[4][t] = r.invalid;
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
      if (t < h) {
        s_min[t] += s_min[t + h];
        s_max[t] += s_max[t + h];
        for (int k = 0; k < 4; ++k) s_cnt[k][t] += s_cnt[k][t + h];
        s_cnt[4][t] |= s_cnt[4][t + h];
      }
      __syncthreads();
    }
    if (t == 0)
      out.store(row, RowCache{s_min[0], s_max[0], s_cnt[0][0], s_cnt[1][0], s_cnt[2][0], s_cnt[3][0], s_cnt[4][0]});
    __syncthreads();
  }
}

// Propose (:905-1018) over the candidate list.
__global__ void sc_propose(const int32_t* __restrict__ cand, const int32_t* __restrict__ st,
                           const int32_t* __restrict__ srow, const double* __restrict__ sval,
                           const double* __restrict__ c, const double* __restrict__ l, const double* __restrict__ u,
                           const double* __restrict__ AL, const double* __restrict__ AU,
                           const double* __restrict__ cache_min, const double* __restrict__ cache_max,
                           const int4* __restrict__ counts, const uint8_t* __restrict__ invalid, double tol,
                           double zero_tol, uint8_t* __restrict__ action, double* __restrict__ side,
                           int32_t* __restrict__ owner) {
  const int count = st[kStCand];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    const int j = cand[q];
    const int row = srow[j];
    const double a = sval[j];
    const double lj = l[j], uj = u[j], cj = c[j];
    // _singleton_column_activity_bounds_from_cache (:756-816).
    if (invalid[row]) continue;
    const double tmin = a >= 0.0 ? a * lj : a * uj;
    const double tmax = a >= 0.0 ? a * uj : a * lj;
    if (isnan(tmin) || isnan(tmax)) continue;
    int4 k = counts[row];
    double vmin = cache_min[row], vmax = cache_max[row];
    if (isinf(tmin)) { if (tmin < 0.0) --k.x; else --k.y; } else { vmin -= tmin; }
    if (isinf(tmax)) { if (tmax < 0.0) --k.z; else --k.w; } else { vmax -= tmax; }
    if (k.x < 0 || k.y < 0 || k.z < 0 || k.w < 0 || (k.x > 0 && k.y > 0) || (k.z > 0 && k.w > 0)) continue;
    const double rmin = k.x > 0 ? -INFINITY : (k.y > 0 ? INFINITY : vmin);
    const double rmax = k.z > 0 ? -INFINITY : (k.w > 0 ? INFINITY : vmax);
    if (isnan(rmin) || isnan(rmax)) continue;
    const double lhs = AL[row], rhs = AU[row];
    uint8_t act = kNone;
    double sd = 0.0;
    if (isfinite(lhs) && isfinite(rhs) && fabs(lhs - rhs) <= tol) {
      const double x1 = (rhs - rmin) / a, x2 = (rhs - rmax) / a;
      const double ilb = fmin(x1, x2), iub = fmax(x1, x2);
      const bool above = !isfinite(uj) || iub <= uj + tol;
      const bool below = !isfinite(lj) || ilb >= lj - tol;
      if (!(above || below)) continue;
      act = above && below ? kEliminateFree : (above ? kEliminateFreeAbove : kEliminateFreeBelow);
      sd = rhs;
    } else {
      // _singleton_column_implied_free_from_above / _below (:818-854).
      bool above = true, below = true;
      if (isfinite(uj)) {
        double implied = INFINITY;
        if (a > 0.0 && isfinite(rhs)) implied = (rhs - rmin) / a;
        else if (a < 0.0 && isfinite(lhs)) implied = (lhs - rmax) / a;
        above = implied <= uj + tol;
      }
      if (isfinite(lj)) {
        double implied = -INFINITY;
        if (a > 0.0 && isfinite(lhs)) implied = (lhs - rmax) / a;
        else if (a < 0.0 && isfinite(rhs)) implied = (rhs - rmin) / a;
        below = implied >= lj - tol;
      }
      // _singleton_column_active_side / _ineq_action (:856-903).
      if (above && below) {
        if ((cj > zero_tol && a > 0.0) || (cj < -zero_tol && a < 0.0)) sd = lhs;
        else if ((cj > zero_tol && a < 0.0) || (cj < -zero_tol && a > 0.0)) sd = rhs;
        else sd = isfinite(lhs) ? lhs : rhs;
        if (!isfinite(sd)) continue;
        act = kSetRowSide;
      } else if (((cj < -zero_tol && a > 0.0 && above) || (cj > zero_tol && a < 0.0 && below)) && isfinite(rhs)) {
        act = kTightenLhs;
        sd = rhs;
      } else if (((cj > zero_tol && a > 0.0 && below) || (cj < -zero_tol && a < 0.0 && above)) && isfinite(lhs)) {
        act = kTightenRhs;
        sd = lhs;
      } else {
        continue;
      }
    }
    action[j] = act;
    side[j] = sd;
    atomicMin(owner + row, act == kEliminateFree ? j - INT_MAX : j);
  }
}

// Stage + commit (:1021-1073, :1157-1189) over the claimed rows.  Every read
// is of the owner's own row and column, so the plan is updated in place; the
// row keeps its owner in `owner` only when the owner column is eliminated.
__global__ void sc_stage(const int32_t* __restrict__ rows, int32_t* st, int n, const uint8_t* __restrict__ action,
                         const double* __restrict__ side, const double* __restrict__ sval,
                         const double* __restrict__ c, const double* __restrict__ l, const double* __restrict__ u,
                         double* __restrict__ AL, double* __restrict__ AU, double tol, int32_t* __restrict__ owner,
                         uint8_t* __restrict__ keep_row, uint8_t* __restrict__ keep_col, uint8_t* __restrict__ kind,
                         int32_t* __restrict__ winners, int64_t* __restrict__ contrib_idx,
                         double* __restrict__ contrib_val) {
  const int count = st[kStRows];
  const int stride = gridDim.x * blockDim.x;
  const int top = (count + stride - 1) / stride * stride;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < top; q += stride) {
    int row = -1, j = -1;
    uint8_t k = 0;
    double contrib = 0.0;
    if (q < count) {
      row = rows[q];
      const int key = owner[row];
      j = key < 0 ? key + INT_MAX : key;
      if (j >= 0 && j < n) {
        const uint8_t act = action[j];
        const double lhs = AL[row], rhs = AU[row];
        if (act == kEliminateFree || act == kEliminateFreeAbove || act == kEliminateFreeBelow) {
          const double a = sval[j];
          contrib = c[j] * rhs / a;
          if (act == kEliminateFree) {
            keep_row[row] = 0;
            k = kRowElimDeleted;
          } else {
            const bool above = act == kEliminateFreeAbove;
            const double bound = above ? l[j] : u[j];
            const bool keep_lower = above ? a < 0.0 : a > 0.0;
            const double shifted = rhs - a * bound;
            if (keep_lower) { AL[row] = shifted; AU[row] = INFINITY; }
            else { AL[row] = -INFINITY; AU[row] = shifted; }
            k = kRowElimKept;
          }
          keep_col[j] = 0;
          owner[row] = j;
        } else {
          bool lo = false, hi = false;
          const double sd = side[j];
          if (act == kSetRowSide) {
            lo = !isfinite(lhs) || fabs(lhs - sd) > tol;
            hi = !isfinite(rhs) || fabs(rhs - sd) > tol;
            AL[row] = sd;
            AU[row] = sd;
          } else if (act == kTightenLhs) {
            lo = true;
            AL[row] = rhs;
          } else if (act == kTightenRhs) {
            hi = true;
            AU[row] = lhs;
          }
          atomicOr(st + kStSide, 1);
          if (lo || hi) k = kRowDualShift;
          owner[row] = kUnclaimed;
        }
      } else {
        owner[row] = kUnclaimed;
      }
      if (k) kind[row] = k;
    }
    const bool elim = k == kRowElimKept || k == kRowElimDeleted;
    const int pe = block_append(st + kStElim, elim);
    if (elim) { contrib_idx[pe] = j; contrib_val[pe] = contrib; }
    const int pw = block_append(st + kStWin, k != 0);
    if (k) winners[pw] = row;
  }
}

// Columns whose cost changes: the live columns of eliminated rows, each
// claimed once through a byte flag.
__global__ void sc_touch(const int32_t* __restrict__ winners, const int32_t* __restrict__ st,
                         const uint8_t* __restrict__ kind, const offset_t* __restrict__ ptr,
                         const int32_t* __restrict__ idx, const uint8_t* __restrict__ keep_col,
                         uint32_t* __restrict__ claimed, int32_t* __restrict__ touched, int32_t* st_w) {
  const int count = st[kStWin];
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < count; w += warps) {
    const int row = winners[w];
    if (kind[row] == kRowDualShift) continue;
    for (offset_t chunk = ptr[row]; chunk < ptr[row + 1]; chunk += 32) {
      const offset_t p = chunk + lane;
      bool take = false;
      int col = 0;
      if (p < ptr[row + 1]) {
        col = idx[p];
        if (keep_col[col]) {
          const uint32_t bit = 1u << (col & 31);
          take = (atomicOr(claimed + (col >> 5), bit) & bit) == 0;
        }
      }
      const int pos = warp_append(st_w + kStTouched, take);
      if (take) touched[pos] = col;
    }
  }
}

// _kernel_apply_singleton_objective_updates_deterministic (:1075-1104): for a
// touched column, c += -(c_o * a / a_o) over its stored entries whose row is
// eliminated by owner o, added in stored order.  Each column belongs to one
// warp and the owners' costs are never touched, so c is updated in place.
__global__ void sc_cost(const int32_t* __restrict__ touched, const int32_t* __restrict__ st, int n,
                        const offset_t* __restrict__ tptr, const int32_t* __restrict__ tidx,
                        const double* __restrict__ tval, const int32_t* __restrict__ owner,
                        const double* __restrict__ sval, double* __restrict__ c) {
  const int count = st[kStTouched];
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < count; w += warps) {
    const int col = touched[w];
    double updated = c[col];
    for (offset_t chunk = tptr[col]; chunk < tptr[col + 1]; chunk += 32) {
      const offset_t p = chunk + lane;
      double term = 0.0;
      bool has = false;
      if (p < tptr[col + 1]) {
        const int o = owner[tidx[p]];
        if (o >= 0 && o < n) {
          has = true;
          term = -(c[o] * tval[p] / sval[o]);
        }
      }
      const unsigned hv = __ballot_sync(0xffffffffu, has);
      for (int k = 0; k < 32; ++k) {
        const double v = __shfl_sync(0xffffffffu, term, k);
        if (hv >> k & 1u) updated += v;
      }
    }
    if (lane == 0) c[col] = updated;
  }
}

// Substitution record sizes (:1191-1284): pivot and live support of each
// eliminated row, in ascending row order.
__global__ void sc_sub_sizes(const int32_t* __restrict__ sorted_rows, int count, const int32_t* __restrict__ owner,
                             const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                             const double* __restrict__ val, const uint8_t* __restrict__ keep_col, double zero_tol,
                             int32_t* __restrict__ sel, int64_t* __restrict__ support) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < count; w += warps) {
    const int row = sorted_rows[w];
    const int col = owner[row];
    int cnt = 0;
    double pivot = 0.0;
    for (offset_t p = ptr[row] + lane; p < ptr[row + 1]; p += 32) {
      const int rc = idx[p];
      if (rc == col) pivot = val[p];
      else if (keep_col[rc]) ++cnt;
    }
    for (int off = 16; off > 0; off >>= 1) {
      cnt += __shfl_down_sync(0xffffffffu, cnt, off);
      const double other = __shfl_down_sync(0xffffffffu, pivot, off);
      if (other != 0.0) pivot = other;
    }
    if (lane == 0) {
      const bool ok = !(fabs(pivot) <= zero_tol);
      sel[w] = ok ? 1 : 0;
      support[w] = ok ? cnt : 0;
    }
  }
}

// SingletonColumnSubstitution records: indices [col, row, count, support...],
// values [pivot, side, l, u, c, row_deleted, coefficients...]; the support
// keeps the stored order (warp ballot compaction).
__global__ void sc_sub_pack(const int32_t* __restrict__ sorted_rows, int count, const int32_t* __restrict__ owner,
                            const uint8_t* __restrict__ kind, const int32_t* __restrict__ sel,
                            const int32_t* __restrict__ rec, const int64_t* __restrict__ spos,
                            const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            const double* __restrict__ val, const uint8_t* __restrict__ keep_col,
                            const double* __restrict__ side, const double* __restrict__ c,
                            const double* __restrict__ l, const double* __restrict__ u, int32_t* __restrict__ types,
                            int64_t* __restrict__ is, int64_t* __restrict__ vs, int32_t* __restrict__ oidx,
                            double* __restrict__ oval) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < count; w += warps) {
    if (!sel[w]) continue;
    const int row = sorted_rows[w];
    const int col = owner[row];
    const int64_t r = rec[w];
    const int64_t s0 = spos[w], s1 = spos[w + 1];
    const int64_t i0 = 3 * r + s0, v0 = 6 * r + s0;
    if (lane == 0) {
      if (r == 0) { is[0] = 0; vs[0] = 0; }
      types[r] = 2;  // SingletonColumnSubstitution
      is[r + 1] = 3 * (r + 1) + s1;
      vs[r + 1] = 6 * (r + 1) + s1;
      oidx[i0] = col;
      oidx[i0 + 1] = row;
      oidx[i0 + 2] = int32_t(s1 - s0);
      oval[v0 + 1] = side[col];
      oval[v0 + 2] = l[col];
      oval[v0 + 3] = u[col];
      oval[v0 + 4] = c[col];
      oval[v0 + 5] = kind[row] == kRowElimDeleted ? 1.0 : 0.0;
    }
    int64_t out = 0;
    for (offset_t chunk = ptr[row]; chunk < ptr[row + 1]; chunk += 32) {
      const offset_t p = chunk + lane;
      bool take = false;
      int rc = -1;
      double a = 0.0;
      if (p < ptr[row + 1]) {
        rc = idx[p];
        a = val[p];
        if (rc == col) oval[v0] = a;
        else take = keep_col[rc] != 0;
      }
      const unsigned mask = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int64_t o = out + __popc(mask & ((1u << lane) - 1u));
        oidx[i0 + 3 + o] = rc;
        oval[v0 + 6 + o] = a;
      }
      out += __popc(mask);
    }
  }
}

// RowDualShift records (:459-508): index [row], value 0.0.
__global__ void sc_shift_pack(const int32_t* __restrict__ sorted_rows, int count, int32_t* __restrict__ types,
                              int64_t* __restrict__ is, int64_t* __restrict__ vs, int32_t* __restrict__ oidx,
                              double* __restrict__ oval) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < count; r += gridDim.x * blockDim.x) {
    if (r == 0) { is[0] = 0; vs[0] = 0; }
    types[r] = 10;  // RowDualShift
    is[r + 1] = r + 1;
    vs[r + 1] = r + 1;
    oidx[r] = sorted_rows[r];
    oval[r] = 0.0;
  }
}

__global__ void sc_fill_i32(int32_t* p, int n, int32_t v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// Sort key: substitution rows first, then dual-shift rows, each ascending.
__global__ void sc_winner_keys(const int32_t* __restrict__ winners, int count, const uint8_t* __restrict__ kind,
                               uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    const int row = winners[q];
    keys[q] = (uint64_t(kind[row] == kRowDualShift ? 1 : 0) << 32) | uint32_t(row);
    vals[q] = row;
  }
}

}  // namespace

void rule_singleton_columns(Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded || !p.enable_singleton_columns) return;
  const int m = lp.m(), n = lp.n();
  if (m == 0 || n == 0) return;
  auto s = ctx().stream;
  Status st;
  st.clear(kStWords);
  DBuf<int32_t> owner(size_t(m), s), cand(size_t(n), s), rows(size_t(m), s), long_rows(size_t(m), s);
  GPP_LAUNCH(sc_fill_i32, grid_stride_blocks(m), kThreads, 0, s, owner.p, m, kUnclaimed);
  GPP_LAUNCH_BYTES(sc_candidates, double(n) * 11 + 16.0 * n, grid_stride_blocks(n), kThreads, 0, s, n, m,
                   plan.keep_col.p, plan.keep_row.p, stats.singleton_col.p, stats.scol_row.p, stats.scol_val.p,
                   stats.row_nnz.p, plan.c.p, plan.l.p, plan.u.p, plan.AL.p, plan.AU.p, p.zero_tol, owner.p, cand.p,
                   rows.p, long_rows.p, st.d);
  const int32_t* f = st.read(4);
  if (f[kStUnbounded]) { plan.has_unbounded = true; return; }
  const int ncand = f[kStCand], nrows = f[kStRows];
  if (ncand == 0) return;

  // Activity cache of the claimed rows.
  DBuf<double> fmin(size_t(m), s), fmax(size_t(m), s);
  DBuf<int4> counts(size_t(m), s);
  DBuf<uint8_t> invalid(size_t(m), s);
  const CacheOut cache{fmin.p, fmax.p, counts.p, invalid.p};
  const int warp_blocks = std::max(1, std::min((nrows + 31) / 32, kNumSMs * 16));
  GPP_LAUNCH(sc_cache_rows, warp_blocks, kThreads, 0, s, rows.p, st.d, stats.row_nnz.p, lp.A.ptr, lp.A.idx,
             lp.A.val, plan.keep_col.p, plan.l.p, plan.u.p, cache);
  if (f[kStLong])
    GPP_LAUNCH(sc_cache_long, std::min(f[kStLong], kNumSMs * 8), kThreads, 0, s, long_rows.p, st.d, stats.row_nnz.p,
               lp.A.ptr, lp.A.idx, lp.A.val, plan.keep_col.p, plan.l.p, plan.u.p, cache);

  // Propose and stage.
  DBuf<uint8_t> action(size_t(n), s), kind(size_t(m), s);
  DBuf<double> side(size_t(n), s), contrib_val(size_t(nrows), s);
  DBuf<int64_t> contrib_idx(size_t(nrows), s);
  DBuf<int32_t> winners(size_t(nrows), s);
  GPP_LAUNCH(sc_propose, grid_stride_blocks(ncand), kThreads, 0, s, cand.p, st.d, stats.scol_row.p,
             stats.scol_val.p, plan.c.p, plan.l.p, plan.u.p, plan.AL.p, plan.AU.p, fmin.p, fmax.p, counts.p,
             invalid.p, p.bound_tol, p.zero_tol, action.p, side.p, owner.p);
  GPP_LAUNCH(sc_stage, grid_stride_blocks(nrows), kThreads, 0, s, rows.p, st.d, n, action.p, side.p,
             stats.scol_val.p, plan.c.p, plan.l.p, plan.u.p, plan.AL.p, plan.AU.p, p.bound_tol, owner.p,
             plan.keep_row.p, plan.keep_col.p, kind.p, winners.p, contrib_idx.p, contrib_val.p);
  f = st.read(kStWords);
  const int nwin = f[kStWin], nelim = f[kStElim];
  const bool any_side = f[kStSide] != 0;
  if (nelim == 0 && !any_side) return;

  // Cost update of the columns sharing an eliminated row.
  if (nelim) {
    DBuf<uint32_t> claimed(size_t(n + 31) / 32, s);
    claimed.zero();
    DBuf<int32_t> touched(size_t(n), s);
    GPP_LAUNCH(sc_touch, std::max(1, std::min((nwin + 7) / 8, kNumSMs * 16)), kThreads, 0, s, winners.p, st.d,
               kind.p, lp.A.ptr, lp.A.idx, plan.keep_col.p, claimed.p, touched.p, st.d);
    const int ntouched = st.read(kStWords)[kStTouched];
    if (ntouched)
      GPP_LAUNCH(sc_cost, std::max(1, std::min((ntouched + 7) / 8, kNumSMs * 16)), kThreads, 0, s, touched.p, st.d,
                 n, lp.AT.ptr, lp.AT.idx, lp.AT.val, owner.p, stats.scol_val.p, plan.c.p);
  }

  // Records, in ascending row order: substitutions, then dual shifts.
  if (p.record_postsolve_tape && nwin) {
    DBuf<uint64_t> keys(size_t(nwin), s);
    DBuf<int32_t> sorted(size_t(nwin), s);
    GPP_LAUNCH(sc_winner_keys, grid_stride_blocks(nwin), kThreads, 0, s, winners.p, nwin, kind.p, keys.p, sorted.p);
    radix_sort_pairs(keys.p, sorted.p, nwin, s);
    const int nshift = nwin - nelim;
    if (nelim) {
      DBuf<int32_t> sel(size_t(nelim) + 1, s), rec(size_t(nelim) + 1, s);
      DBuf<int64_t> sup(size_t(nelim) + 1, s), spos(size_t(nelim) + 1, s);
      const int blocks = std::max(1, std::min((nelim + 7) / 8, kNumSMs * 16));
      GPP_LAUNCH(sc_sub_sizes, blocks, kThreads, 0, s, sorted.p, nelim, owner.p, lp.A.ptr, lp.A.idx, lp.A.val,
                 plan.keep_col.p, p.zero_tol, sel.p, sup.p);
      exclusive_scan_i32(sel.p, rec.p, nelim, s);
      exclusive_scan_i64(sup.p, spos.p, nelim, s);
      const auto [recs32, support] = read_scalars(rec.p + nelim, spos.p + nelim);
      const int64_t recs = recs32;
      if (recs) {
        PostsolveSegment seg = make_segment(recs, 3 * recs + support, 6 * recs + support);
        GPP_LAUNCH(sc_sub_pack, blocks, kThreads, 0, s, sorted.p, nelim, owner.p, kind.p, sel.p, rec.p, spos.p,
                   lp.A.ptr, lp.A.idx, lp.A.val, plan.keep_col.p, side.p, plan.c.p, plan.l.p, plan.u.p,
                   seg.types.p, seg.is.p, seg.vs.p, seg.idx.p, seg.val.p);
        plan.tape.push_back(std::move(seg));
      }
    }
    if (nshift) {
      PostsolveSegment seg = make_segment(nshift, nshift, nshift);
      GPP_LAUNCH(sc_shift_pack, grid_stride_blocks(nshift), kThreads, 0, s, sorted.p + nelim, nshift, seg.types.p,
                 seg.is.p, seg.vs.p, seg.idx.p, seg.val.p);
      plan.tape.push_back(std::move(seg));
    }
  }

  if (nelim) {
    auto [ci, cv] = to_host2(contrib_idx.p, size_t(nelim), contrib_val.p, size_t(nelim));
    std::vector<std::pair<int64_t, double>> entries(ci.size());
    for (size_t k = 0; k < ci.size(); ++k) entries[k] = {ci[k], cv[k]};
    plan.obj_delta += det_sum_sparse(std::move(entries));
  }
  plan.has_row_action = true;
  plan.has_col_action = plan.has_col_action || nelim > 0;
  plan.has_change = true;
}

}  // namespace gpp
