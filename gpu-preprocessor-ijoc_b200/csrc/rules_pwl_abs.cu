// Structure-specific Startup rule: piecewise-linear reformulation of absolute
// values (reference rules/rule_piecewise_linear_reformulation_absolute_value.cu,
// entry apply_rule_... at :2425-2728, prefix screen :2389-2424).
//
// An epigraph pair is two rows with exactly two stored entries on the same
// columns (t, e) that read  a t - a e >= 0  and  a t + a e >= 0  (a > 0; a
// row (-inf, 0] counts as its negation), i.e. t >= |e|.  Three model layouts
// are recognised, each all-or-nothing: any mismatch leaves the model as it is.
//  * l1 split, m = 3k.  Block i is rows 3i (an equality holding e once and t
//    never) and 3i+1, 3i+2 (the epigraph pair).  e is split as e = p - q with
//    p on t's column and q on e's column, both in [0, inf): the equality gets
//    e's coefficient on p and its negation on q, the costs become c_t + c_e
//    and c_t - c_e, and the pair rows go, except that the first is kept as
//    l_e <= p - q <= u_e when e had a finite bound and the residual-bound mode
//    preserves it (:470-617, :619-657).
//  * graph l1, m = 4k.  Block i is an equality, the epigraph pair, and a row
//    s - beta t >= 0.  The same split with costs c_t +- c_e / rho; every other
//    row of t must be such a row whose auxiliary s has zero cost, no upper
//    bound and only such rows: those rows and s go, and postsolve sets
//    s = max(l_s, max beta t) (:756-1205, :2002-2240).
//  * outer pair + linked l1.  A prefix of 3-row groups
//    b - f >= 0, b + f >= 0, f - b >= 0  forces a free column f equal to a
//    column b in [0, u]: f is replaced by b everywhere and its cost added to
//    b's.  Then 8-row blocks: an equality holding e, the pair q >= |e|, the
//    link  alpha q - s = 0  and four rows  x - s >= 0.  e is split on (q, e),
//    s = alpha (p + q) is substituted into the four rows and the pair and link
//    rows go (:1207-1660, :2502-2700).
// Every decision the reference takes on exact coefficient identities and
// incidence counts is taken here on the same quantities, so the same models
// are accepted and the rewritten matrices, costs and recovery data are equal.
// Work is data-parallel throughout: per-block validation kernels chained on
// one device status word (a failed step makes the rest return at once, so a
// chain costs one readback), warp-per-row rewrites, and sorted groups where
// the reference runs a serial loop (the outer pairs' cost accumulation keeps
// the pair order within each bounded column).
#include "engine.cuh"
#include "sort.hpp"

namespace gpp {

namespace {

constexpr double kCoefTol = 1.0e-12;   // ABSOLUTE_VALUE_COEFFICIENT_TOL (:25)
constexpr int32_t kUnassigned = -1, kBoundRole = -2, kBlockRole = -3, kAuxRole = -2;
enum : uint8_t { kEqRow = 1, kEqZeroTwo = 2, kLowerTwo = 4, kZeroSidedTwo = 8 };

// A row's side flags and, for rows with exactly two stored entries, those
// entries in column order (raw, and as the zero-sided form z1 x1 + z2 x2 >= 0
// when the row is [0, inf) or (-inf, 0]); _kernel_structural_row_metadata
// (:271-353).
struct PairRow {
  int32_t c1, c2;
  double v1, v2, z1, z2;
  uint32_t flags;
};

__device__ PairRow pair_row(int row, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            const double* __restrict__ val, const double* __restrict__ AL,
                            const double* __restrict__ AU) {
  PairRow r{-1, -1, 0.0, 0.0, 0.0, 0.0, 0u};
  const double al = AL[row], au = AU[row];
  const bool eq = isfinite(al) && isfinite(au) && al == au;
  if (eq) r.flags |= kEqRow;
  const offset_t lo = ptr[row];
  if (ptr[row + 1] - lo != 2) return r;
  int32_t c1 = idx[lo], c2 = idx[lo + 1];
  double v1 = val[lo], v2 = val[lo + 1];
  if (c2 < c1) {
    const int32_t tc = c1; c1 = c2; c2 = tc;
    const double tv = v1; v1 = v2; v2 = tv;
  }
  r.c1 = c1; r.c2 = c2; r.v1 = v1; r.v2 = v2;
  if (eq && al == 0.0) r.flags |= kEqZeroTwo;
  if (isfinite(al) && isinf(au) && au > 0.0) r.flags |= kLowerTwo;
  const bool zero_lower = al == 0.0 && isinf(au) && au > 0.0;
  const bool zero_upper = isinf(al) && al < 0.0 && au == 0.0;
  if (zero_lower || zero_upper) {
    const double s = zero_lower ? 1.0 : -1.0;
    r.flags |= kZeroSidedTwo;
    r.z1 = s * v1;
    r.z2 = s * v2;
  }
  return r;
}

__global__ void row_metadata(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                             const double* __restrict__ val, const double* __restrict__ AL,
                             const double* __restrict__ AU, PairRow* __restrict__ rows) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    rows[i] = pair_row(i, ptr, idx, val, AL, AU);
}

__device__ __forceinline__ bool zero_sided(const PairRow& r) { return (r.flags & kZeroSidedTwo) != 0; }

// t >= |e| from two zero-sided rows on the same columns
// (_sls_extract_l1_split_pair_device, :205-241).
__device__ bool epigraph_pair(const PairRow& a, const PairRow& b, int32_t* t, int32_t* e) {
  if (a.c1 != b.c1 || a.c2 != b.c2) return false;
  if (isfinite(a.z1) && a.z1 > 0.0 && a.z1 == b.z1 && a.z2 == -a.z1 && b.z2 == b.z1) {
    *t = a.c1;
    *e = a.c2;
    return *t != *e;
  }
  if (isfinite(a.z2) && a.z2 > 0.0 && a.z2 == b.z2 && a.z1 == -a.z2 && b.z1 == b.z2) {
    *t = a.c2;
    *e = a.c1;
    return *t != *e;
  }
  return false;
}

// The graph variant's orientation (_sls_extract_l1_orientation_device,
// :243-269): the second row's coefficients are read on the first row's
// columns, and rho = |e coefficient / t coefficient| of the first row.
__device__ bool epigraph_orientation(const PairRow& a, const PairRow& b, int32_t* t, int32_t* e, double* rho) {
  PairRow bb = b;
  bb.c1 = a.c1;
  bb.c2 = a.c2;
  if (!epigraph_pair(a, bb, t, e)) return false;
  if (*t == a.c1 && *e == a.c2) *rho = fabs(a.z2 / a.z1);
  else if (*t == a.c2 && *e == a.c1) *rho = fabs(a.z1 / a.z2);
  else *rho = 0.0;
  return isfinite(*rho) && *rho > 0.0;
}

// The three-group signature of one outer pair (_sls_outer_pair_signature_device).
__device__ bool outer_signature(const PairRow& a, const PairRow& b, const PairRow& c) {
  if (a.c1 != b.c1 || a.c1 != c.c1 || a.c2 != b.c2 || a.c2 != c.c2) return false;
  return a.z1 == 1.0 && a.z2 == -1.0 && b.z1 == 1.0 && b.z2 == 1.0 && c.z1 == -1.0 && c.z2 == 1.0;
}

__device__ __forceinline__ void fail(int32_t* status) { atomicMax(status, 1); }

// ---- prefix screen (:2389-2424) -------------------------------------------------

__global__ void prefix_screen(int m, int n, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                              const double* __restrict__ val, const double* __restrict__ AL,
                              const double* __restrict__ AU, int32_t* __restrict__ out) {
  if (blockIdx.x || threadIdx.x) return;
  PairRow r[4];
  for (int i = 0; i < 4; ++i) r[i] = i < m ? pair_row(i, ptr, idx, val, AL, AU) : PairRow{-1, -1, 0, 0, 0, 0, 0u};
  int32_t t, e;
  auto l1_pair = [&](const PairRow& a, const PairRow& b) {
    return zero_sided(a) && zero_sided(b) && epigraph_pair(a, b, &t, &e);
  };
  // Zero-sided coefficients of a row that is not zero-sided read as 0 and
  // its columns as -1, as the reference's prefix rows do.
  auto zc1 = [](const PairRow& a) { return zero_sided(a) ? a.c1 : -1; };
  auto zc2 = [](const PairRow& a) { return zero_sided(a) ? a.c2 : -1; };
  const bool graph = m >= 4 && m % 4 == 0 && (r[0].flags & kEqRow) && l1_pair(r[1], r[2]) && zero_sided(r[3]) &&
                     (r[3].z1 > kCoefTol || r[3].z2 > kCoefTol) && (r[3].z1 < -kCoefTol || r[3].z2 < -kCoefTol) &&
                     (zc1(r[3]) == zc1(r[1]) || zc1(r[3]) == zc2(r[1]) || zc2(r[3]) == zc1(r[1]) ||
                      zc2(r[3]) == zc2(r[1]));
  const bool outer = m >= 11 && zero_sided(r[0]) && zero_sided(r[1]) && zero_sided(r[2]) &&
                     outer_signature(r[0], r[1], r[2]);
  const bool split = m >= 3 && m % 3 == 0 && (r[0].flags & kEqRow) && l1_pair(r[1], r[2]);
  *out = m > 0 && n > 0 && (graph || outer || split) ? 1 : 0;
}

// ---- rewritten matrices ---------------------------------------------------------

// Row pointers from per-row counts; returns the matrix with idx/val allocated.
DevCsr alloc_rows(int m, int n, const int32_t* counts, cudaStream_t s) {
  DevCsr out;
  out.rows = m;
  out.cols = n;
  out.ptr = dalloc<offset_t>(size_t(m) + 1);
  exclusive_scan_i32(counts, out.ptr, m, s);
  out.nnz = read_scalar(out.ptr + m);
  out.idx = dalloc<int32_t>(size_t(out.nnz));
  out.val = dalloc<double>(size_t(out.nnz));
  return out;
}

// Warp-per-row rewrite of a strictly sorted row that holds `e` once and
// `t` never: e's entry is dropped and (t, w), (e, -w) inserted in column
// order, w = e's coefficient divided by rho when rho != 1 is given
// (_kernel_..._split_fill :677-754, _kernel_structural_graph_fill :1139-1205).
// Entry p lands at  (p - lo) - [p after e] + [col > t] + [col > e].
__device__ void split_row(int lane, offset_t lo, offset_t hi, const int32_t* __restrict__ idx,
                          const double* __restrict__ val, int32_t t, int32_t e, const double* rho, offset_t w0,
                          int32_t* __restrict__ oidx, double* __restrict__ oval) {
  offset_t pe = hi;
  for (offset_t b = lo; b < hi; b += 32) {
    const offset_t p = b + lane;
    const unsigned hit = __ballot_sync(0xffffffffu, p < hi && idx[p] == e);
    if (hit) { pe = b + __ffs(hit) - 1; break; }
  }
  double w = pe < hi ? val[pe] : 0.0;
  if (rho) w = w / *rho;
  const int32_t first = t < e ? t : e, second = t < e ? e : t;
  const double first_v = t < e ? w : -w, second_v = t < e ? -w : w;
  int32_t below_first = 0, below_second = 0;
  for (offset_t p = lo + lane; p < hi; p += 32) {
    if (p == pe) continue;
    const int32_t col = idx[p];
    const offset_t dst = w0 + (p - lo) - (p > pe ? 1 : 0) + (col > first ? 1 : 0) + (col > second ? 1 : 0);
    oidx[dst] = col;
    oval[dst] = val[p];
    below_first += col < first ? 1 : 0;
    below_second += col < second ? 1 : 0;
  }
  below_first = __reduce_add_sync(0xffffffffu, below_first);
  below_second = __reduce_add_sync(0xffffffffu, below_second);
  if (lane == 0) {
    oidx[w0 + below_first] = first;
    oval[w0 + below_first] = first_v;
    oidx[w0 + below_second + 1] = second;
    oval[w0 + below_second + 1] = second_v;
  }
}

// Are the rows strictly ascending?  (_kernel_structural_check_csr_sorted)
__global__ void rows_ascending(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                               int32_t* __restrict__ bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    for (offset_t p = ptr[i] + 1; p < ptr[i + 1]; ++p)
      if (idx[p - 1] >= idx[p]) { atomicMax(bad, 1); break; }
}
__global__ void row_sort_keys(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                              uint64_t* __restrict__ keys, int32_t* __restrict__ pos) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  for (int i = warp; i < m; i += (gridDim.x * blockDim.x) >> 5)
    for (offset_t p = ptr[i] + lane; p < ptr[i + 1]; p += 32) {
      keys[p] = (uint64_t(uint32_t(i)) << 32) | uint32_t(idx[p]);
      pos[p] = p;
    }
}
__global__ void row_sort_gather(offset_t nnz, const uint64_t* __restrict__ keys, const int32_t* __restrict__ pos,
                                const double* __restrict__ val, int32_t* __restrict__ oidx,
                                double* __restrict__ oval) {
  for (offset_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += gridDim.x * blockDim.x) {
    oidx[q] = int32_t(uint32_t(keys[q] & 0xffffffffu));
    oval[q] = val[pos[q]];
  }
}

// Sorts every row by column (a stable sort by (row, column)) unless already
// ascending; false when a row then holds a column twice
// (ensure_structural_csr_rows_sorted_unique, :107-174).
bool sort_rows_unique(DevCsr& M, Status& st, cudaStream_t s) {
  if (M.rows <= 0 || M.nnz <= 0) return true;
  st.clear(1);
  GPP_LAUNCH(rows_ascending, grid_stride_blocks(M.rows), kThreads, 0, s, M.rows, M.ptr, M.idx, st.d);
  if (st.read(1)[0] == 0) return true;
  DBuf<uint64_t> keys(size_t(M.nnz), s);
  DBuf<int32_t> pos(size_t(M.nnz), s);
  GPP_LAUNCH(row_sort_keys, grid_stride_blocks(int64_t(M.rows) * 32), kThreads, 0, s, M.rows, M.ptr, M.idx, keys.p,
             pos.p);
  radix_sort_pairs(keys.p, pos.p, M.nnz, s);
  DBuf<double> vals(size_t(M.nnz), s);
  vals.copy_from(M.val, size_t(M.nnz));
  GPP_LAUNCH(row_sort_gather, grid_stride_blocks(M.nnz), kThreads, 0, s, M.nnz, keys.p, pos.p, vals.p, M.idx, M.val);
  st.clear(1);
  GPP_LAUNCH(rows_ascending, grid_stride_blocks(M.rows), kThreads, 0, s, M.rows, M.ptr, M.idx, st.d);
  return st.read(1)[0] == 0;
}

__global__ void fill_i32(int32_t* p, int64_t n, int32_t v) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = v;
}
__global__ void fill_f64(double* p, int64_t n, double v) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = v;
}

// ---- shared by the split and graph variants --------------------------------------

// Every t and e column has one owner (_kernel_..._split_claim_roles, :442-468).
__global__ void claim_roles(int blocks, int n, const int32_t* __restrict__ t_cols, const int32_t* __restrict__ e_cols,
                            int32_t* __restrict__ owner, int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
    const int32_t t = t_cols[b], e = e_cols[b];
    if (t < 0 || t >= n || e < 0 || e >= n || t == e) { fail(status); continue; }
    if (atomicCAS(owner + t, kUnassigned, 2 * b) != kUnassigned) fail(status);
    if (atomicCAS(owner + e, kUnassigned, 2 * b + 1) != kUnassigned) fail(status);
  }
}

// ---- l1 split ----------------------------------------------------------------------

__global__ void split_extract(int blocks, const PairRow* __restrict__ rows, int32_t* __restrict__ t_cols,
                              int32_t* __restrict__ e_cols, int32_t* __restrict__ status) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
    const PairRow& eq = rows[3 * b];
    const PairRow r1 = rows[3 * b + 1], r2 = rows[3 * b + 2];
    int32_t t = -1, e = -1;
    if (!(eq.flags & kEqRow) || !zero_sided(r1) || !zero_sided(r2) || !epigraph_pair(r1, r2, &t, &e)) {
      fail(status);
      continue;
    }
    t_cols[b] = t;
    e_cols[b] = e;
  }
}

struct SplitArgs {
  const uint8_t *keep_row, *keep_col;
  const double *c, *l, *u;
  const offset_t* a_ptr;
  const int32_t* a_idx;
  const double* a_val;
  const offset_t* at_ptr;
  const int32_t* at_idx;
  const double* at_val;
  const int32_t *t_cols, *e_cols;
  int mode;
  double as_free_min;
};

// _kernel_..._split_validate_blocks (:470-617).
__global__ void split_validate(int blocks, SplitArgs g, uint8_t* __restrict__ preserve, int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
    preserve[b] = 0;
    const int32_t t = g.t_cols[b], e = g.e_cols[b];
    const int eq = 3 * b, r1 = eq + 1, r2 = eq + 2;
    const double l_t = g.l[t], u_t = g.u[t], l_e = g.l[e], u_e = g.u[e], c_t = g.c[t], c_e = g.c[e];
    const bool t_ok = l_t == 0.0 && isinf(u_t) && u_t > 0.0;
    const bool e_ok = !isnan(l_e) && !isnan(u_e) && !(isinf(l_e) && l_e > 0.0) && !(isinf(u_e) && u_e < 0.0) &&
                      l_e <= u_e;
    const bool e_free = isinf(l_e) && l_e < 0.0 && isinf(u_e) && u_e > 0.0;
    const bool preserve_mode = g.mode == GPP_RESIDUAL_PRESERVE_FINITE;
    const bool strict_mode = g.mode == GPP_RESIDUAL_STRICT_FREE_ONLY;
    const bool legacy_mode = g.mode == GPP_RESIDUAL_LEGACY_WIDE_AS_FREE;
    const bool legacy_free = legacy_mode && isfinite(g.as_free_min) && g.as_free_min > 0.0 &&
                             l_e <= -g.as_free_min && u_e >= g.as_free_min;
    const bool mode_ok = preserve_mode || strict_mode || legacy_mode;
    const bool residual_ok = e_free || preserve_mode || legacy_free;
    bool costs_ok = isfinite(c_t) && isfinite(c_e);
    if (costs_ok) costs_ok = isfinite(c_t + c_e) && isfinite(c_t - c_e);
    if (!t_ok || !e_ok || !costs_ok || !g.keep_row[eq] || !g.keep_row[r1] || !g.keep_row[r2] || !g.keep_col[t] ||
        !g.keep_col[e] || !mode_ok || !residual_ok) {
      fail(status);
      continue;
    }
    // Exact incidence: e once in the equality (strictly ascending, finite,
    // nonzero entries) and once in each pair row; t only in the pair rows.
    int a_t = 0, a_e = 0, prev = -1;
    bool ok = true;
    for (offset_t p = g.a_ptr[eq]; p < g.a_ptr[eq + 1]; ++p) {
      const int32_t col = g.a_idx[p];
      if (col <= prev || !isfinite(g.a_val[p]) || g.a_val[p] == 0.0) ok = false;
      prev = col;
      a_t += col == t;
      a_e += col == e;
    }
    ok = ok && a_t == 0 && a_e == 1;
    int t1 = 0, t2 = 0;
    for (offset_t p = g.at_ptr[t]; p < g.at_ptr[t + 1]; ++p) {
      if (fabs(g.at_val[p]) <= kCoefTol) { ok = false; continue; }
      const int32_t row = g.at_idx[p];
      if (row == r1) ++t1; else if (row == r2) ++t2; else ok = false;
    }
    int e0 = 0, e1 = 0, e2 = 0;
    for (offset_t p = g.at_ptr[e]; p < g.at_ptr[e + 1]; ++p) {
      if (fabs(g.at_val[p]) <= kCoefTol) { ok = false; continue; }
      const int32_t row = g.at_idx[p];
      if (row == eq) ++e0; else if (row == r1) ++e1; else if (row == r2) ++e2; else ok = false;
    }
    if (!(ok && t1 == 1 && t2 == 1 && e0 == 1 && e1 == 1 && e2 == 1)) { fail(status); continue; }
    preserve[b] = preserve_mode && !e_free ? 1 : 0;
  }
}

__global__ void split_counts(int m, const offset_t* __restrict__ ptr, const uint8_t* __restrict__ preserve,
                             int32_t* __restrict__ counts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const int k = i % 3;
    counts[i] = k == 0 ? ptr[i + 1] - ptr[i] + 1 : (k == 1 && preserve[i / 3] ? 2 : 0);
  }
}

__global__ void split_fill(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ val, const int32_t* __restrict__ t_cols,
                           const int32_t* __restrict__ e_cols, const uint8_t* __restrict__ preserve,
                           const offset_t* __restrict__ optr, int32_t* __restrict__ oidx,
                           double* __restrict__ oval) {
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += (gridDim.x * blockDim.x) >> 5) {
    const int b = i / 3, k = i % 3;
    const int32_t t = t_cols[b], e = e_cols[b];
    if (k == 0) {
      split_row(lane, ptr[i], ptr[i + 1], idx, val, t, e, nullptr, optr[i], oidx, oval);
    } else if (k == 1 && preserve[b] && lane == 0) {
      // The kept bound row  l_e <= p - q <= u_e.
      const offset_t w = optr[i];
      const bool t_first = t < e;
      oidx[w] = t_first ? t : e;
      oval[w] = t_first ? 1.0 : -1.0;
      oidx[w + 1] = t_first ? e : t;
      oval[w + 1] = t_first ? -1.0 : 1.0;
    }
  }
}

// _kernel_..._split_apply_plan (:619-657).
__global__ void split_apply(int blocks, const int32_t* __restrict__ t_cols, const int32_t* __restrict__ e_cols,
                            const uint8_t* __restrict__ preserve, uint8_t* __restrict__ keep_row, double* c,
                            double* l, double* u, double* AL, double* AU) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
    const int32_t t = t_cols[b], e = e_cols[b];
    const int r1 = 3 * b + 1, r2 = r1 + 1;
    const double c_t = c[t], c_e = c[e], l_e = l[e], u_e = u[e];
    if (preserve[b]) {
      AL[r1] = l_e;
      AU[r1] = u_e;
    } else {
      keep_row[r1] = 0;
    }
    keep_row[r2] = 0;
    c[t] = c_t + c_e;
    c[e] = c_t - c_e;
    l[t] = 0.0;
    l[e] = 0.0;
    u[t] = INFINITY;
    u[e] = INFINITY;
  }
}

// ---- graph l1 ------------------------------------------------------------------------

struct GraphArgs {
  const PairRow* rows;
  const offset_t* a_ptr;
  const int32_t* a_idx;
  const double* a_val;
  const offset_t* at_ptr;
  const int32_t* at_idx;
  const double* at_val;
  const double *c, *l, *u, *AL, *AU;
  int m, n;
};

// _kernel_structural_graph_extract_blocks (:756-889).
__global__ void graph_extract(int blocks, GraphArgs g, int32_t* __restrict__ t_cols, int32_t* __restrict__ e_cols,
                              double* __restrict__ rhos, int32_t* __restrict__ status) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
    const int eq = 4 * b;
    const PairRow r1 = g.rows[eq + 1], r2 = g.rows[eq + 2], r3 = g.rows[eq + 3];
    if (!(g.rows[eq].flags & kEqRow) || !zero_sided(r1) || !zero_sided(r2) || !zero_sided(r3)) {
      fail(status);
      continue;
    }
    int32_t t = -1, e = -1;
    double rho = 0.0;
    if (!epigraph_orientation(r1, r2, &t, &e, &rho)) { fail(status); continue; }
    double coeff_t, coeff_s;
    if (r3.c1 == t) { coeff_t = r3.z1; coeff_s = r3.z2; }
    else if (r3.c2 == t) { coeff_t = r3.z2; coeff_s = r3.z1; }
    else { fail(status); continue; }
    if (!(coeff_t < -kCoefTol && coeff_s > kCoefTol)) { fail(status); continue; }
    if (t < 0 || t >= g.n || e < 0 || e >= g.n || t == e) { fail(status); continue; }
    const bool bounds_ok = isinf(g.l[e]) && g.l[e] < 0.0 && isinf(g.u[e]) && g.u[e] > 0.0 && g.l[t] == 0.0 &&
                           isinf(g.u[t]) && g.u[t] > 0.0 && isfinite(g.c[t]) && g.c[t] >= 0.0 && isfinite(g.c[e]);
    bool costs_ok = bounds_ok && isfinite(rho) && rho > 0.0;
    if (costs_ok) {
      const double scaled = g.c[e] / rho;
      costs_ok = isfinite(scaled) && isfinite(g.c[t] + scaled) && isfinite(g.c[t] - scaled);
    }
    if (!bounds_ok || !costs_ok) { fail(status); continue; }
    int e_count = 0, t_count = 0, prev = -1;
    bool row_ok = true;
    for (offset_t p = g.a_ptr[eq]; p < g.a_ptr[eq + 1]; ++p) {
      const int32_t col = g.a_idx[p];
      if (col <= prev || !isfinite(g.a_val[p]) || g.a_val[p] == 0.0) row_ok = false;
      prev = col;
      e_count += col == e;
      t_count += col == t;
    }
    int s0 = 0, s1 = 0, s2 = 0;
    bool at_ok = true;
    for (offset_t p = g.at_ptr[e]; p < g.at_ptr[e + 1]; ++p) {
      const int32_t row = g.at_idx[p];
      if (row == eq) ++s0; else if (row == eq + 1) ++s1; else if (row == eq + 2) ++s2; else at_ok = false;
    }
    if (!(row_ok && e_count == 1 && t_count == 0 && at_ok && s0 == 1 && s1 == 1 && s2 == 1)) {
      fail(status);
      continue;
    }
    t_cols[b] = t;
    e_cols[b] = e;
    rhos[b] = rho;
  }
}

// Every other row of t is  s - beta t >= 0  with its own auxiliary s
// (_kernel_structural_graph_mark_extra_rows, :891-975).
__global__ void graph_mark_rows(int blocks, GraphArgs g, const int32_t* __restrict__ t_cols,
                                int32_t* __restrict__ row_block, int32_t* __restrict__ row_slack,
                                double* __restrict__ row_factor, int32_t* __restrict__ owner,
                                int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
    const int32_t t = t_cols[b];
    const int r1 = 4 * b + 1, r2 = 4 * b + 2;
    for (offset_t p = g.at_ptr[t]; p < g.at_ptr[t + 1]; ++p) {
      const int32_t row = g.at_idx[p];
      if (row == r1 || row == r2) continue;
      bool ok = g.AL[row] == 0.0 && isinf(g.AU[row]) && g.AU[row] > 0.0;
      const offset_t lo = g.a_ptr[row];
      ok = ok && g.a_ptr[row + 1] - lo == 2;
      double coeff_t = 0.0, coeff_s = 0.0;
      int32_t slack = -1;
      if (ok) {
        const int32_t c1 = g.a_idx[lo], c2 = g.a_idx[lo + 1];
        const double v1 = g.a_val[lo], v2 = g.a_val[lo + 1];
        ok = c1 != c2 && isfinite(v1) && isfinite(v2);
        if (ok && c1 == t) { coeff_t = v1; coeff_s = v2; slack = c2; }
        else if (ok && c2 == t) { coeff_t = v2; coeff_s = v1; slack = c1; }
        else ok = false;
      }
      ok = ok && slack >= 0 && slack < g.n && coeff_t < -kCoefTol && coeff_s > kCoefTol;
      const double factor = ok ? -coeff_t / coeff_s : 0.0;
      ok = ok && isfinite(factor) && factor > 0.0;
      if (!ok) { fail(status); continue; }
      const int32_t prior = atomicCAS(row_block + row, -1, b);
      if (prior != -1 && prior != b) { fail(status); continue; }
      row_slack[row] = slack;
      row_factor[row] = factor;
      const int32_t o = atomicCAS(owner + slack, kUnassigned, kAuxRole);
      if (o != kUnassigned && o != kAuxRole) fail(status);
    }
  }
}

// The zero-cost, no-up-lock dual fix of the auxiliaries: every row of an
// auxiliary must be one of the certified rows (_kernel_structural_graph_dual_fix_auxiliaries).
__global__ void graph_aux_rows(GraphArgs g, const int32_t* __restrict__ owner, const int32_t* __restrict__ row_block,
                               const int32_t* __restrict__ row_slack, uint8_t* __restrict__ removable,
                               int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < g.n; j += gridDim.x * blockDim.x) {
    if (owner[j] != kAuxRole) continue;
    bool ok = g.c[j] == 0.0 && !isnan(g.l[j]) && !(isinf(g.l[j]) && g.l[j] > 0.0) && isinf(g.u[j]) && g.u[j] > 0.0;
    for (offset_t p = g.at_ptr[j]; ok && p < g.at_ptr[j + 1]; ++p) {
      const int32_t row = g.at_idx[p];
      ok = row >= 0 && row < g.m && row_block[row] >= 0 && row_slack[row] == j && g.at_val[p] > kCoefTol &&
           g.AL[row] == 0.0 && isinf(g.AU[row]) && g.AU[row] > 0.0;
      if (ok) removable[row] = 1;
    }
    if (!ok) fail(status);
  }
}

// The block's own fourth row is one of them (_kernel_structural_graph_validate_required_rows).
__global__ void graph_required_rows(int blocks, int n, const int32_t* __restrict__ row_block,
                                    const int32_t* __restrict__ row_slack, const double* __restrict__ row_factor,
                                    const uint8_t* __restrict__ removable, int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
    const int r = 4 * b + 3;
    const int32_t slack = row_slack[r];
    const double f = row_factor[r];
    if (row_block[r] != b || slack < 0 || slack >= n || !isfinite(f) || f <= 0.0 || !removable[r]) fail(status);
  }
}

__global__ void graph_counts(int m, const offset_t* __restrict__ ptr, int32_t* __restrict__ counts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    counts[i] = i % 4 == 0 ? ptr[i + 1] - ptr[i] + 1 : 0;
}
__global__ void graph_fill(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ val, const int32_t* __restrict__ t_cols,
                           const int32_t* __restrict__ e_cols, const double* __restrict__ rhos,
                           const offset_t* __restrict__ optr, int32_t* __restrict__ oidx, double* __restrict__ oval) {
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += (gridDim.x * blockDim.x) >> 5) {
    if (i % 4) continue;
    const int b = i / 4;
    split_row(lane, ptr[i], ptr[i + 1], idx, val, t_cols[b], e_cols[b], rhos + b, optr[i], oidx, oval);
  }
}

// _kernel_structural_graph_apply_plan (:1055-1114) and the auxiliaries' removal.
__global__ void graph_apply(int blocks, GraphArgs g, const int32_t* __restrict__ t_cols,
                            const int32_t* __restrict__ e_cols, const double* __restrict__ rhos,
                            const uint8_t* __restrict__ removable, uint8_t* __restrict__ keep_row, double* c, double* l,
                            double* u, int32_t* __restrict__ status) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
    const int r1 = 4 * b + 1, r2 = r1 + 1;
    const int32_t t = t_cols[b], e = e_cols[b];
    keep_row[r1] = 0;
    keep_row[r2] = 0;
    bool ok = true;
    for (offset_t p = g.at_ptr[t]; p < g.at_ptr[t + 1]; ++p) {
      const int32_t row = g.at_idx[p];
      if (row == r1 || row == r2) continue;
      if (removable[row]) keep_row[row] = 0;
      else { ok = false; break; }
    }
    if (!ok) { fail(status); continue; }
    const double inv_rho = 1.0 / rhos[b];
    const double c_t = c[t], c_e = c[e];
    c[t] = c_t + c_e * inv_rho;
    c[e] = c_t - c_e * inv_rho;
    l[t] = 0.0;
    l[e] = 0.0;
    u[t] = INFINITY;
    u[e] = INFINITY;
  }
}
__global__ void drop_aux(int n, const int32_t* __restrict__ owner, uint8_t* __restrict__ keep_col) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    if (owner[j] == kAuxRole) keep_col[j] = 0;
}

// Max-slack groups: one per auxiliary, ordered by its first removable row,
// entries in row order (capture_absolute_value_max_slacks_device,
// device_recovery.cu:698-748).
__global__ void slack_first_row(int m, const int32_t* __restrict__ row_block, const int32_t* __restrict__ row_slack,
                                const uint8_t* __restrict__ removable, int32_t* __restrict__ first) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
    if (removable[r] && row_block[r] >= 0 && row_slack[r] >= 0) atomicMin(first + row_slack[r], r);
}
__global__ void slack_flags(int m, const int32_t* __restrict__ row_block, const int32_t* __restrict__ row_slack,
                            const uint8_t* __restrict__ removable, int32_t* __restrict__ flag) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
    flag[r] = removable[r] && row_block[r] >= 0 && row_slack[r] >= 0 ? 1 : 0;
}
__global__ void slack_keys(int m, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                           const int32_t* __restrict__ row_slack, const int32_t* __restrict__ first,
                           uint64_t* __restrict__ keys, int32_t* __restrict__ rows) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
    if (flag[r]) {
      keys[pos[r]] = (uint64_t(uint32_t(first[row_slack[r]])) << 32) | uint32_t(r);
      rows[pos[r]] = r;
    }
}
__global__ void slack_heads(int k, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < k; q += gridDim.x * blockDim.x)
    head[q] = q == 0 || (keys[q] >> 32) != (keys[q - 1] >> 32) ? 1 : 0;
}
__global__ void slack_pack(int k, const uint64_t* __restrict__ keys, const int32_t* __restrict__ rows,
                           const int32_t* __restrict__ head, const int32_t* __restrict__ hpos,
                           const int32_t* __restrict__ t_cols, const int32_t* __restrict__ row_block,
                           const int32_t* __restrict__ row_slack, const double* __restrict__ row_factor,
                           int32_t* __restrict__ slack, int32_t* __restrict__ start, int32_t* __restrict__ t_out,
                           double* __restrict__ f_out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < k; q += gridDim.x * blockDim.x) {
    const int r = rows[q];
    if (head[q]) {
      slack[hpos[q]] = row_slack[r];
      start[hpos[q]] = q;
    }
    if (q == k - 1) start[hpos[k]] = k;
    t_out[q] = t_cols[row_block[r]];
    f_out[q] = row_factor[r];
  }
}

// ---- outer pair + linked l1 ------------------------------------------------------------

// Leading run of valid 3-row pair groups (_kernel_structural_outer_count_pairs):
// the first invalid group index, by atomicMin.
__global__ void outer_first_bad(int groups, const PairRow* __restrict__ rows, int32_t* __restrict__ first_bad) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
    const PairRow a = rows[3 * q], b = rows[3 * q + 1], c = rows[3 * q + 2];
    if (!(zero_sided(a) && zero_sided(b) && zero_sided(c) && outer_signature(a, b, c))) atomicMin(first_bad, q);
  }
}

struct OuterArgs {
  const PairRow* rows;
  const offset_t* a_ptr;
  const int32_t* a_idx;
  const double *c, *l, *u;
  int n, start_row, pairs, blocks;
};

// Per pair: bounds and costs, and one owner per free column
// (_kernel_structural_outer_validate_pairs_and_build_free_to_bound, first loop).
__global__ void outer_pairs_check(OuterArgs g, int32_t* __restrict__ free_to_bound, uint64_t* __restrict__ keys,
                                  int32_t* __restrict__ vals, int32_t* __restrict__ status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.pairs; i += gridDim.x * blockDim.x) {
    const PairRow& r = g.rows[3 * i];
    const int32_t b = r.c1, f = r.c2;
    keys[i] = (uint64_t(uint32_t(b < 0 ? 0 : b)) << 32) | uint32_t(i);
    vals[i] = i;
    if (b < 0 || b >= g.n || f < 0 || f >= g.n || b == f || g.l[b] != 0.0 || !isfinite(g.u[b]) || g.u[b] < 0.0 ||
        !isinf(g.l[f]) || g.l[f] >= 0.0 || !isinf(g.u[f]) || g.u[f] <= 0.0 || !isfinite(g.c[b]) ||
        !isfinite(g.c[f])) {
      fail(status);
      continue;
    }
    if (atomicCAS(free_to_bound + f, kUnassigned, b) != kUnassigned) fail(status);
  }
}

// The bounded column's cost plus its free columns' costs in pair order (the
// reference's serial loop restricted to each bounded column); every partial
// sum finite.
__global__ void outer_pair_costs(OuterArgs g, const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals,
                                 double* __restrict__ bound_cost, int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < g.pairs; q += gridDim.x * blockDim.x) {
    const uint32_t b = uint32_t(keys[q] >> 32);
    if (q > 0 && uint32_t(keys[q - 1] >> 32) == b) continue;
    double acc = g.c[b];
    bool ok = true;
    for (int k = q; k < g.pairs && uint32_t(keys[k] >> 32) == b; ++k) {
      acc += g.c[g.rows[3 * vals[k]].c2];
      if (!isfinite(acc)) ok = false;
    }
    if (!ok) fail(status);
    bound_cost[b] = acc;
  }
}

// No bounded column is also a free one; then mark the bounded role
// (second loop of the same kernel).
__global__ void outer_bound_check(OuterArgs g, const int32_t* __restrict__ free_to_bound, int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.pairs; i += gridDim.x * blockDim.x)
    if (free_to_bound[g.rows[3 * i].c1] >= 0) fail(status);
}
__global__ void outer_bound_mark(OuterArgs g, int32_t* __restrict__ free_to_bound, const int32_t* __restrict__ status) {
  if (*(volatile const int32_t*)status) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.pairs; i += gridDim.x * blockDim.x)
    free_to_bound[g.rows[3 * i].c1] = kBoundRole;
}

__device__ __forceinline__ int32_t outer_map(const int32_t* free_to_bound, int32_t col) {
  const int32_t b = free_to_bound[col];
  return b >= 0 ? b : col;
}

// _kernel_structural_outer_extract_blocks (:1264-1381).
__global__ void outer_extract(OuterArgs g, const int32_t* __restrict__ free_to_bound, int32_t* __restrict__ q_cols,
                              int32_t* __restrict__ e_cols, int32_t* __restrict__ s_cols, double* __restrict__ alphas,
                              int32_t* __restrict__ x_cols, int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.blocks; b += gridDim.x * blockDim.x) {
    const int dense = g.start_row + 8 * b;
    const PairRow ep1 = g.rows[dense + 1], ep2 = g.rows[dense + 2], link = g.rows[dense + 3];
    if (!(g.rows[dense].flags & kEqRow) || !zero_sided(ep1) || !zero_sided(ep2) || !(link.flags & kEqZeroTwo)) {
      fail(status);
      continue;
    }
    // The pair reads  -e + q >= 0,  e + q >= 0  on (e, q) in column order
    // (_sls_extract_l1_pair_device).
    if (!(ep1.z1 == -1.0 && ep1.z2 == 1.0 && ep2.z1 == 1.0 && ep2.z2 == 1.0) || ep1.c2 == ep1.c1) {
      fail(status);
      continue;
    }
    const int32_t e = ep1.c1, q = ep1.c2;
    int32_t s;
    double alpha;
    if (link.c1 == q) {
      s = link.c2;
      alpha = link.v1;
      if (link.v2 != -1.0) { fail(status); continue; }
    } else if (link.c2 == q) {
      s = link.c1;
      alpha = link.v2;
      if (link.v1 != -1.0) { fail(status); continue; }
    } else {
      fail(status);
      continue;
    }
    if (!isfinite(alpha) || alpha <= 0.0 || q == e) { fail(status); continue; }
    bool ok = true;
    for (int k = 0; k < 4 && ok; ++k) {
      const PairRow loc = g.rows[dense + 4 + k];
      if (!(loc.flags & kLowerTwo)) { ok = false; break; }
      int32_t x;
      if (loc.c1 == s) {
        if (loc.v1 != -1.0 || loc.v2 != 1.0) { ok = false; break; }
        x = loc.c2;
      } else if (loc.c2 == s) {
        if (loc.v2 != -1.0 || loc.v1 != 1.0) { ok = false; break; }
        x = loc.c1;
      } else {
        ok = false;
        break;
      }
      const int32_t mx = outer_map(free_to_bound, x);
      if (mx == q || mx == e) { ok = false; break; }
      x_cols[4 * b + k] = x;
    }
    if (!ok) { fail(status); continue; }
    q_cols[b] = q;
    e_cols[b] = e;
    s_cols[b] = s;
    alphas[b] = alpha;
  }
}

// Each q, e and s has one owner and is no outer endpoint
// (_kernel_structural_outer_mark_block_roles).
__global__ void outer_roles(OuterArgs g, const int32_t* __restrict__ q_cols, const int32_t* __restrict__ e_cols,
                            const int32_t* __restrict__ s_cols, int32_t* __restrict__ free_to_bound,
                            int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 3 * g.blocks; k += gridDim.x * blockDim.x) {
    const int b = k / 3, which = k % 3;
    const int32_t col = which == 0 ? q_cols[b] : which == 1 ? e_cols[b] : s_cols[b];
    if (col < 0 || col >= g.n) { fail(status); continue; }
    if (atomicCAS(free_to_bound + col, kUnassigned, kBlockRole) != kUnassigned) fail(status);
  }
}
// No x column is another block's q, e or s (_kernel_structural_outer_validate_local_x_roles).
__global__ void outer_x_roles(OuterArgs g, const int32_t* __restrict__ free_to_bound,
                              const int32_t* __restrict__ x_cols, int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 4 * g.blocks; k += gridDim.x * blockDim.x) {
    const int32_t x = x_cols[k];
    if (x < 0 || x >= g.n || free_to_bound[x] == kBlockRole) fail(status);
  }
}
// _kernel_structural_outer_block_validate (:1463-1544).
__global__ void outer_block_check(OuterArgs g, const int32_t* __restrict__ free_to_bound,
                                  const int32_t* __restrict__ q_cols, const int32_t* __restrict__ e_cols,
                                  const int32_t* __restrict__ s_cols, const double* __restrict__ alphas,
                                  const int32_t* __restrict__ x_cols, int32_t* __restrict__ status) {
  if (*(volatile int32_t*)status) return;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.blocks; b += gridDim.x * blockDim.x) {
    const int32_t q = q_cols[b], e = e_cols[b], s = s_cols[b];
    if (q < 0 || q >= g.n || e < 0 || e >= g.n || s < 0 || s >= g.n) { fail(status); continue; }
    const bool bounds_ok = isinf(g.l[e]) && g.l[e] < 0.0 && isinf(g.u[e]) && g.u[e] > 0.0 && g.l[q] == 0.0 &&
                           isinf(g.u[q]) && g.u[q] > 0.0 && g.l[s] == 0.0 && isinf(g.u[s]) && g.u[s] > 0.0 &&
                           isfinite(g.c[q]) && isfinite(g.c[e]) && isfinite(g.c[s]);
    const double alpha = alphas[b];
    bool costs_ok = bounds_ok && isfinite(alpha) && alpha > 0.0;
    if (costs_ok) {
      const double linked = alpha * g.c[s];
      costs_ok = isfinite(linked) && isfinite(g.c[q] + g.c[e] + linked) && isfinite(g.c[q] - g.c[e] + linked);
    }
    if (!bounds_ok || !costs_ok) { fail(status); continue; }
    bool ok = true;
    for (int k = 0; k < 4; ++k) {
      const int32_t x = x_cols[4 * b + k];
      if (x < 0 || x >= g.n ||
          !(g.l[x] == 0.0 && isinf(g.u[x]) && g.u[x] > 0.0 && isfinite(g.c[x]) && g.c[x] > kCoefTol)) {
        ok = false;
        break;
      }
    }
    if (!ok) { fail(status); continue; }
    const int dense = g.start_row + 8 * b;
    int e_seen = 0;
    for (offset_t p = g.a_ptr[dense]; p < g.a_ptr[dense + 1]; ++p) {
      const int32_t col = g.a_idx[p];
      if (free_to_bound[col] == kBlockRole) {
        if (col != e) { ok = false; break; }
        ++e_seen;
      }
    }
    if (!ok || e_seen != 1) fail(status);
  }
}

__global__ void outer_counts(int m, int start_row, const offset_t* __restrict__ ptr, int32_t* __restrict__ counts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const int k = (i - start_row) % 8;
    counts[i] = i >= start_row && (k == 0 || k >= 4) ? ptr[i + 1] - ptr[i] + 1 : 0;
  }
}
// Dense row: e -> (q: a, e: -a) at e's place; local rows: s -> (q, e) both
// alpha * a; every other column through the outer map (_kernel_structural_outer_fill,
// :1608-1666).  Columns are ordered afterwards when the mapping disturbed them.
__global__ void outer_fill(int m, int start_row, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ val, const int32_t* __restrict__ free_to_bound,
                           const int32_t* __restrict__ q_cols, const int32_t* __restrict__ e_cols,
                           const int32_t* __restrict__ s_cols, const double* __restrict__ alphas,
                           const offset_t* __restrict__ optr, int32_t* __restrict__ oidx, double* __restrict__ oval) {
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += (gridDim.x * blockDim.x) >> 5) {
    if (i < start_row) continue;
    const int k = (i - start_row) % 8;
    if (!(k == 0 || k >= 4)) continue;
    const int b = (i - start_row) / 8;
    const int32_t q = q_cols[b], e = e_cols[b], s = s_cols[b];
    const double alpha = alphas[b];
    const int32_t special = k == 0 ? e : s;
    const offset_t lo = ptr[i], hi = ptr[i + 1];
    offset_t ps = hi;
    for (offset_t base = lo; base < hi; base += 32) {
      const offset_t p = base + lane;
      const unsigned hit = __ballot_sync(0xffffffffu, p < hi && idx[p] == special);
      if (hit) { ps = base + __ffs(hit) - 1; break; }
    }
    const bool q_first = q < e;
    for (offset_t p = lo + lane; p < hi; p += 32) {
      const offset_t dst = optr[i] + (p - lo) + (p > ps ? 1 : 0);
      const int32_t col = idx[p];
      const double v = val[p];
      if (p == ps) {
        const double a = k == 0 ? v : v * alpha;
        oidx[dst] = q_first ? q : e;
        oval[dst] = k == 0 ? (q_first ? a : -a) : a;
        oidx[dst + 1] = q_first ? e : q;
        oval[dst + 1] = k == 0 ? (q_first ? -a : a) : a;
      } else {
        oidx[dst] = outer_map(free_to_bound, col);
        oval[dst] = v;
      }
    }
  }
}

// _kernel_structural_outer_pair_apply and _block_apply (:1437-1585).
__global__ void outer_pair_apply(OuterArgs g, const double* __restrict__ bound_cost, uint8_t* __restrict__ keep_row,
                                 uint8_t* __restrict__ keep_col, double* __restrict__ c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.pairs; i += gridDim.x * blockDim.x) {
    const PairRow& r = g.rows[3 * i];
    keep_row[3 * i] = 0;
    keep_row[3 * i + 1] = 0;
    keep_row[3 * i + 2] = 0;
    keep_col[r.c2] = 0;
    c[r.c1] = bound_cost[r.c1];
  }
}
__global__ void outer_block_apply(OuterArgs g, const int32_t* __restrict__ q_cols, const int32_t* __restrict__ e_cols,
                                  const int32_t* __restrict__ s_cols, const double* __restrict__ alphas,
                                  uint8_t* __restrict__ keep_row, uint8_t* __restrict__ keep_col, double* c, double* l,
                                  double* u) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.blocks; b += gridDim.x * blockDim.x) {
    const int dense = g.start_row + 8 * b;
    const int32_t q = q_cols[b], e = e_cols[b], s = s_cols[b];
    const double alpha = alphas[b];
    keep_row[dense + 1] = 0;
    keep_row[dense + 2] = 0;
    keep_row[dense + 3] = 0;
    keep_col[s] = 0;
    const double c_e = c[e], c_q = c[q], c_s = c[s];
    c[q] = c_e + c_q + alpha * c_s;
    c[e] = -c_e + c_q + alpha * c_s;
    l[q] = 0.0;
    l[e] = 0.0;
    u[q] = INFINITY;
    u[e] = INFINITY;
  }
}
__global__ void outer_pair_ids(int pairs, const PairRow* __restrict__ rows, int32_t* __restrict__ bound,
                               int32_t* __restrict__ free_col) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += gridDim.x * blockDim.x) {
    bound[i] = rows[3 * i].c1;
    free_col[i] = rows[3 * i].c2;
  }
}

// ---- the three attempts ---------------------------------------------------------------

struct Ctx {
  Plan& plan;
  const WorkingLp& lp;
  const gpp_params& p;
  DBuf<PairRow>& rows;
  Status& st;
  cudaStream_t s;
};

void set_changed(Plan& plan, DevCsr&& A) {
  plan.new_A = A;
  plan.has_new_A = true;
  plan.has_change = true;
  plan.has_col_action = true;
  plan.has_row_action = true;
}

std::unique_ptr<AbsValueRecovery> splits_recovery(int32_t pattern, const int32_t* t, const int32_t* e,
                                                  const double* rho, int count, cudaStream_t s) {
  auto r = std::make_unique<AbsValueRecovery>();
  r->pattern = pattern;
  r->splits = count;
  r->split_t.alloc(size_t(count), s);
  r->split_e.alloc(size_t(count), s);
  r->split_rho.alloc(size_t(count), s);
  r->split_t.copy_from(t, size_t(count));
  r->split_e.copy_from(e, size_t(count));
  if (rho) r->split_rho.copy_from(rho, size_t(count));
  else GPP_LAUNCH(fill_f64, grid_stride_blocks(count), kThreads, 0, s, r->split_rho.p, count, 1.0);
  return r;
}

// try_apply_l1_split (:1871-2000).
bool try_split(Ctx& x) {
  const DevCsr& A = x.lp.A;
  const int m = A.rows, n = A.cols;
  if (m < 3 || m % 3 || x.plan.has_new_A) return false;
  const int blocks = m / 3;
  auto s = x.s;
  DBuf<int32_t> t(size_t(blocks), s), e(size_t(blocks), s), owner(size_t(n), s);
  DBuf<uint8_t> preserve(size_t(blocks), s);
  x.st.clear(1);
  const int gb = grid_stride_blocks(blocks);
  GPP_LAUNCH(split_extract, gb, kThreads, 0, s, blocks, x.rows.p, t.p, e.p, x.st.d);
  GPP_LAUNCH(fill_i32, grid_stride_blocks(n), kThreads, 0, s, owner.p, n, kUnassigned);
  GPP_LAUNCH(claim_roles, gb, kThreads, 0, s, blocks, n, t.p, e.p, owner.p, x.st.d);
  const SplitArgs g{x.plan.keep_row.p, x.plan.keep_col.p, x.plan.c.p, x.plan.l.p, x.plan.u.p, A.ptr, A.idx, A.val,
                    x.lp.AT.ptr, x.lp.AT.idx, x.lp.AT.val, t.p, e.p,
                    int(x.p.piecewise_linear_reformulation_absolute_value_residual_bound_mode),
                    x.p.piecewise_linear_reformulation_absolute_value_residual_bound_as_free_min};
  GPP_LAUNCH(split_validate, gb, kThreads, 0, s, blocks, g, preserve.p, x.st.d);
  if (x.st.read(1)[0]) return false;
  DBuf<int32_t> counts(size_t(m) + 1, s);
  GPP_LAUNCH(split_counts, grid_stride_blocks(m), kThreads, 0, s, m, A.ptr, preserve.p, counts.p);
  DevCsr out = alloc_rows(m, n, counts.p, s);
  GPP_LAUNCH(split_fill, grid_stride_blocks(int64_t(m) * 32), kThreads, 0, s, m, A.ptr, A.idx, A.val, t.p, e.p,
             preserve.p, out.ptr, out.idx, out.val);
  GPP_LAUNCH(split_apply, gb, kThreads, 0, s, blocks, t.p, e.p, preserve.p, x.plan.keep_row.p, x.plan.c.p,
             x.plan.l.p, x.plan.u.p, x.plan.AL.p, x.plan.AU.p);
  set_changed(x.plan, std::move(out));
  x.plan.absval = splits_recovery(GPP_ABS_L1_SPLIT, t.p, e.p, nullptr, blocks, s);
  return true;
}

// try_apply_graph_l1 (:2002-2245).
bool try_graph(Ctx& x) {
  const DevCsr& A = x.lp.A;
  const int m = A.rows, n = A.cols;
  if (m < 4 || m % 4 || x.plan.has_new_A) return false;
  const int blocks = m / 4;
  auto s = x.s;
  const GraphArgs g{x.rows.p, A.ptr, A.idx, A.val, x.lp.AT.ptr, x.lp.AT.idx, x.lp.AT.val, x.plan.c.p, x.plan.l.p,
                    x.plan.u.p, x.plan.AL.p, x.plan.AU.p, m, n};
  DBuf<int32_t> t(size_t(blocks), s), e(size_t(blocks), s), owner(size_t(n), s);
  DBuf<double> rho(size_t(blocks), s);
  DBuf<int32_t> row_block(size_t(m), s), row_slack(size_t(m), s);
  DBuf<double> row_factor(size_t(m), s);
  DBuf<uint8_t> removable(size_t(m), s);
  const int gb = grid_stride_blocks(blocks), gm = grid_stride_blocks(m);
  x.st.clear(1);
  GPP_LAUNCH(graph_extract, gb, kThreads, 0, s, blocks, g, t.p, e.p, rho.p, x.st.d);
  GPP_LAUNCH(fill_i32, grid_stride_blocks(n), kThreads, 0, s, owner.p, n, kUnassigned);
  GPP_LAUNCH(claim_roles, gb, kThreads, 0, s, blocks, n, t.p, e.p, owner.p, x.st.d);
  GPP_LAUNCH(fill_i32, gm, kThreads, 0, s, row_block.p, m, -1);
  GPP_LAUNCH(fill_i32, gm, kThreads, 0, s, row_slack.p, m, -1);
  row_factor.zero();
  removable.zero();
  GPP_LAUNCH(graph_mark_rows, gb, kThreads, 0, s, blocks, g, t.p, row_block.p, row_slack.p, row_factor.p, owner.p,
             x.st.d);
  GPP_LAUNCH(graph_aux_rows, grid_stride_blocks(n), kThreads, 0, s, g, owner.p, row_block.p, row_slack.p,
             removable.p, x.st.d);
  GPP_LAUNCH(graph_required_rows, gb, kThreads, 0, s, blocks, n, row_block.p, row_slack.p, row_factor.p,
             removable.p, x.st.d);
  if (x.st.read(1)[0]) return false;
  DBuf<int32_t> counts(size_t(m) + 1, s);
  GPP_LAUNCH(graph_counts, gm, kThreads, 0, s, m, A.ptr, counts.p);
  DevCsr out = alloc_rows(m, n, counts.p, s);
  GPP_LAUNCH(graph_fill, grid_stride_blocks(int64_t(m) * 32), kThreads, 0, s, m, A.ptr, A.idx, A.val, t.p, e.p,
             rho.p, out.ptr, out.idx, out.val);
  GPP_LAUNCH(graph_apply, gb, kThreads, 0, s, blocks, g, t.p, e.p, rho.p, removable.p, x.plan.keep_row.p,
             x.plan.c.p, x.plan.l.p, x.plan.u.p, x.st.d);
  GPP_LAUNCH(drop_aux, grid_stride_blocks(n), kThreads, 0, s, n, owner.p, x.plan.keep_col.p);
  if (x.st.read(1)[0]) {
    // Not reachable for a model that passed validation; the plan is then
    // discarded by the caller (has_change stays false).
    free_csr(out);
    return false;
  }
  set_changed(x.plan, std::move(out));
  auto r = splits_recovery(GPP_ABS_GRAPH_L1, t.p, e.p, rho.p, blocks, s);
  // Max-slack groups.
  DBuf<int32_t> first(size_t(n), s), flag(size_t(m) + 1, s), pos(size_t(m) + 1, s);
  GPP_LAUNCH(fill_i32, grid_stride_blocks(n), kThreads, 0, s, first.p, n, INT32_MAX);
  GPP_LAUNCH(slack_first_row, gm, kThreads, 0, s, m, row_block.p, row_slack.p, removable.p, first.p);
  GPP_LAUNCH(slack_flags, gm, kThreads, 0, s, m, row_block.p, row_slack.p, removable.p, flag.p);
  exclusive_scan_i32(flag.p, pos.p, m, s);
  const int k = read_scalar(pos.p + m);
  if (k > 0) {
    DBuf<uint64_t> keys(size_t(k), s);
    DBuf<int32_t> rows(size_t(k), s), head(size_t(k) + 1, s), hpos(size_t(k) + 1, s);
    GPP_LAUNCH(slack_keys, gm, kThreads, 0, s, m, flag.p, pos.p, row_slack.p, first.p, keys.p, rows.p);
    radix_sort_pairs(keys.p, rows.p, k, s);
    GPP_LAUNCH(slack_heads, grid_stride_blocks(k), kThreads, 0, s, k, keys.p, head.p);
    exclusive_scan_i32(head.p, hpos.p, k, s);
    const int groups = read_scalar(hpos.p + k);
    r->max_groups = groups;
    r->max_entries = k;
    r->max_slack.alloc(size_t(groups), s);
    r->max_start.alloc(size_t(groups) + 1, s);
    r->max_t.alloc(size_t(k), s);
    r->max_factor.alloc(size_t(k), s);
    GPP_LAUNCH(slack_pack, grid_stride_blocks(k), kThreads, 0, s, k, keys.p, rows.p, head.p, hpos.p, t.p,
               row_block.p, row_slack.p, row_factor.p, r->max_slack.p, r->max_start.p, r->max_t.p, r->max_factor.p);
  }
  x.plan.absval = std::move(r);
  return true;
}

// The outer-pair branch of apply_rule_... (:2502-2700).  Returns true when
// the model was rewritten or the rewrite was rejected after the blocks
// matched (duplicate columns after the mapping), i.e. when the graph variant
// is not to be tried.
bool try_outer(Ctx& x, bool* changed) {
  *changed = false;
  const DevCsr& A = x.lp.A;
  const int m = A.rows, n = A.cols;
  auto s = x.s;
  const int groups = m / 3;
  DBuf<int32_t> first_bad(1, s);
  GPP_LAUNCH(fill_i32, 1, 32, 0, s, first_bad.p, 1, groups);
  GPP_LAUNCH(outer_first_bad, grid_stride_blocks(groups), kThreads, 0, s, groups, x.rows.p, first_bad.p);
  const int pairs = read_scalar(first_bad.p);
  const int start_row = 3 * pairs;
  if (pairs == 0 || start_row >= m || (m - start_row) % 8) return false;
  const int blocks = (m - start_row) / 8;
  const OuterArgs g{x.rows.p, A.ptr, A.idx, x.plan.c.p, x.plan.l.p, x.plan.u.p, n, start_row, pairs, blocks};
  DBuf<int32_t> free_to_bound(size_t(n), s), vals(size_t(pairs), s);
  DBuf<uint64_t> keys(size_t(pairs), s);
  DBuf<double> bound_cost(size_t(n), s);
  DBuf<int32_t> q(size_t(blocks), s), e(size_t(blocks), s), sc(size_t(blocks), s), xc(size_t(4) * blocks, s);
  DBuf<double> alpha(size_t(blocks), s);
  const int gp = grid_stride_blocks(pairs), gb = grid_stride_blocks(blocks);
  GPP_LAUNCH(fill_i32, grid_stride_blocks(n), kThreads, 0, s, free_to_bound.p, n, kUnassigned);
  x.st.clear(1);
  GPP_LAUNCH(outer_pairs_check, gp, kThreads, 0, s, g, free_to_bound.p, keys.p, vals.p, x.st.d);
  radix_sort_pairs(keys.p, vals.p, pairs, s);
  GPP_LAUNCH(outer_pair_costs, gp, kThreads, 0, s, g, keys.p, vals.p, bound_cost.p, x.st.d);
  GPP_LAUNCH(outer_bound_check, gp, kThreads, 0, s, g, free_to_bound.p, x.st.d);
  GPP_LAUNCH(outer_bound_mark, gp, kThreads, 0, s, g, free_to_bound.p, x.st.d);
  GPP_LAUNCH(outer_extract, gb, kThreads, 0, s, g, free_to_bound.p, q.p, e.p, sc.p, alpha.p, xc.p, x.st.d);
  GPP_LAUNCH(outer_roles, grid_stride_blocks(int64_t(3) * blocks), kThreads, 0, s, g, q.p, e.p, sc.p,
             free_to_bound.p, x.st.d);
  GPP_LAUNCH(outer_x_roles, grid_stride_blocks(int64_t(4) * blocks), kThreads, 0, s, g, free_to_bound.p, xc.p,
             x.st.d);
  GPP_LAUNCH(outer_block_check, gb, kThreads, 0, s, g, free_to_bound.p, q.p, e.p, sc.p, alpha.p, xc.p, x.st.d);
  if (x.st.read(1)[0]) return false;
  DBuf<int32_t> counts(size_t(m) + 1, s);
  GPP_LAUNCH(outer_counts, grid_stride_blocks(m), kThreads, 0, s, m, start_row, A.ptr, counts.p);
  DevCsr out = alloc_rows(m, n, counts.p, s);
  GPP_LAUNCH(outer_fill, grid_stride_blocks(int64_t(m) * 32), kThreads, 0, s, m, start_row, A.ptr, A.idx, A.val,
             free_to_bound.p, q.p, e.p, sc.p, alpha.p, out.ptr, out.idx, out.val);
  if (!sort_rows_unique(out, x.st, s)) {
    free_csr(out);
    return true;
  }
  GPP_LAUNCH(outer_pair_apply, gp, kThreads, 0, s, g, bound_cost.p, x.plan.keep_row.p, x.plan.keep_col.p,
             x.plan.c.p);
  GPP_LAUNCH(outer_block_apply, gb, kThreads, 0, s, g, q.p, e.p, sc.p, alpha.p, x.plan.keep_row.p,
             x.plan.keep_col.p, x.plan.c.p, x.plan.l.p, x.plan.u.p);
  set_changed(x.plan, std::move(out));
  auto r = splits_recovery(GPP_ABS_OUTER_PAIR, q.p, e.p, nullptr, blocks, s);
  r->pairs = pairs;
  r->pair_bound.alloc(size_t(pairs), s);
  r->pair_free.alloc(size_t(pairs), s);
  GPP_LAUNCH(outer_pair_ids, gp, kThreads, 0, s, pairs, x.rows.p, r->pair_bound.p, r->pair_free.p);
  r->links = blocks;
  r->link_slack.alloc(size_t(blocks), s);
  r->link_t.alloc(size_t(blocks), s);
  r->link_factor.alloc(size_t(blocks), s);
  r->link_slack.copy_from(sc.p, size_t(blocks));
  r->link_t.copy_from(q.p, size_t(blocks));
  r->link_factor.copy_from(alpha.p, size_t(blocks));
  x.plan.absval = std::move(r);
  *changed = true;
  return true;
}

}  // namespace

bool absolute_value_prefix_screen(const WorkingLp& lp) {
  if (lp.m() <= 0 || lp.n() <= 0) return false;
  auto s = ctx().stream;
  Status st;
  st.clear(1);
  GPP_LAUNCH(prefix_screen, 1, 32, 0, s, lp.m(), lp.n(), lp.A.ptr, lp.A.idx, lp.A.val, lp.AL, lp.AU, st.d);
  return st.read(1)[0] != 0;
}

void rule_absolute_value(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded || !p.enable_piecewise_linear_reformulation_absolute_value) return;
  const int m = lp.A.rows, n = lp.A.cols;
  if (m < 3 || n < 2) return;
  auto s = ctx().stream;
  DBuf<PairRow> rows(size_t(m), s);
  GPP_LAUNCH(row_metadata, grid_stride_blocks(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, lp.A.val, plan.AL.p,
             plan.AU.p, rows.p);
  Status st;
  Ctx x{plan, lp, p, rows, st, s};
  if (try_split(x)) return;
  bool changed = false;
  if (try_outer(x, &changed)) return;
  try_graph(x);
}

}  // namespace gpp
