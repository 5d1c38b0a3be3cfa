// Structure-specific Startup rule: column domination on strict unit
// set-covering LPs (reference rule_column_domination.cu:1-386).
//
// The model qualifies only if every row is  sum x >= 1  (AL = 1, AU = +inf)
// with a column of cost exactly 1 in it, every column is a [0, 1] variable
// with a positive integer cost, and every stored coefficient (of A and of
// A^T) is exactly 1.  Then a column whose cost exceeds its number of rows is
// dominated: the cost-1 columns of its rows cover them for no more, so it is
// fixed at 0 and removed.  The rule applies only when at least
// max(1, column_domination_min_fixed_cols) columns qualify and they are at
// least column_domination_min_candidate_ratio of all columns.  The
// reference's sampled probe is a prefilter of the same checks and changes no
// result, so it is not repeated here.
//
// Projected auxiliaries (reference rule_two_row_variable_elimination.cu and
// rule_zero_cost_product_variables.cu): a zero-cost column whose only live
// rows certify it can be recovered from the others is removed with those
// rows, and a projected-column record (type 14) rebuilds it in postsolve as
// the maximum of its lower expressions.
//   * Two-row variable elimination: a zero-cost column with finite bounds in
//     exactly two live one-sided rows of at most 8 live entries, one row a
//     lower and one an upper bound on it, with a strictly positive
//     interval-certificate margin between the two row envelopes and the box.
//   * Zero-cost product variables: a [0, 1] zero-cost column z in exactly
//     three live rows forming the McCormick envelope z >= x + y - 1,
//     z <= x, z <= y of two other [0, 1] columns.
// Both select only candidates whose rows no other candidate uses (and, for
// products, whose endpoints are not candidates), and apply past a minimum
// count and share of the live columns.
#include "engine.cuh"

namespace gpp {

namespace {

enum : int32_t { kBadRow = 1, kBadColumn = 2, kBadValue = 4, kNoWitness = 8 };

// First the cheap checks (row sides, column boxes and costs: m + n reads),
// which reject almost every model; only then the per-entry ones (every
// coefficient of A and A^T, and a cost-1 witness in each row).
__global__ void cd_validate_sides(int m, int n, const double* __restrict__ c, const double* __restrict__ AL,
                                  const double* __restrict__ AU, const double* __restrict__ l,
                                  const double* __restrict__ u, int32_t* __restrict__ failure) {
  int32_t bad = 0;
  const int stride = gridDim.x * blockDim.x;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
    const double cj = c[j];
    if (l[j] != 0.0 || u[j] != 1.0 || !(isfinite(cj) && cj >= 1.0 && floor(cj) == cj)) bad |= kBadColumn;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    if (AL[i] != 1.0 || !(isinf(AU[i]) && AU[i] > 0.0)) bad |= kBadRow;
  bad = __reduce_or_sync(0xffffffffu, bad);
  if (bad && (threadIdx.x & 31) == 0) atomicOr(failure, bad);
}

__global__ void cd_validate_entries(int m, offset_t nnz, const offset_t* __restrict__ ptr,
                                    const int32_t* __restrict__ idx, const double* __restrict__ a,
                                    const double* __restrict__ at, const double* __restrict__ c,
                                    int32_t* __restrict__ failure) {
  int32_t bad = 0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nnz; t += stride)
    if (a[t] != 1.0 || at[t] != 1.0) bad |= kBadValue;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += stride) {
    bool witness = false;
    for (offset_t p = ptr[i]; p < ptr[i + 1] && !witness; ++p) witness = c[idx[p]] == 1.0;
    if (!witness) bad |= kNoWitness;
  }
  bad = __reduce_or_sync(0xffffffffu, bad);
  if (bad && (threadIdx.x & 31) == 0) atomicOr(failure, bad);
}

// Cost above degree: dominated.  Counted per block, one atomic per block.
__global__ void cd_mark(int n, const offset_t* __restrict__ at_ptr, const double* __restrict__ c,
                        uint8_t* __restrict__ dominated, int32_t* __restrict__ count) {
  const int stride = gridDim.x * blockDim.x;
  const int top = (n + stride - 1) / stride * stride;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < top; j += stride) {
    bool d = false;
    if (j < n) {
      d = c[j] > double(at_ptr[j + 1] - at_ptr[j]);
      dominated[j] = d ? 1 : 0;
    }
    block_append(count, d);
  }
}

__global__ void cd_apply(int n, const uint8_t* __restrict__ dominated, uint8_t* __restrict__ keep_col,
                         double* __restrict__ l, double* __restrict__ u) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    if (dominated[j]) {
      keep_col[j] = 0;
      l[j] = 0.0;
      u[j] = 0.0;
    }
}

// ---- projected auxiliaries ----------------------------------------------

constexpr int kMaxCertifiedRowNnz = 8;
constexpr int kMaxAffineTerms = kMaxCertifiedRowNnz - 1;
constexpr int kMaxDifferenceTerms = 2 * kMaxAffineTerms;
constexpr int kFmeCol = 14;

struct Affine {
  double constant;
  int length;
  int32_t cols[kMaxAffineTerms];
  double coeffs[kMaxAffineTerms];
};

__device__ __forceinline__ bool neg_inf(double v) { return isinf(v) && v < 0.0; }
__device__ __forceinline__ bool pos_inf(double v) { return isinf(v) && v > 0.0; }

// A row with one finite side bounds the pivot column from below (lower) or
// above; `bound` is the finite side.
__device__ bool one_sided(double al, double au, double pivot, double zero_tol, bool* lower, double* bound) {
  if (!isfinite(pivot) || fabs(pivot) <= zero_tol) return false;
  if (isfinite(al) && pos_inf(au)) { *lower = pivot > 0.0; *bound = al; return true; }
  if (neg_inf(al) && isfinite(au)) { *lower = pivot < 0.0; *bound = au; return true; }
  return false;
}

// Adds coeff * x_col to a short expression, merging a repeated column.
__device__ bool add_term(int32_t col, double coeff, int32_t* cols, double* coeffs, int* length, int capacity) {
  if (!isfinite(coeff)) return false;
  for (int k = 0; k < *length; ++k)
    if (cols[k] == col) {
      coeffs[k] += coeff;
      return isfinite(coeffs[k]);
    }
  if (*length >= capacity) return false;
  cols[*length] = col;
  coeffs[*length] = coeff;
  ++*length;
  return true;
}

// x_col >= (or <=) bound / pivot - sum_{k != col} a_k / pivot x_k over the
// live entries of `row` (2..max_row_nnz of them, the pivot exactly once).
__device__ bool row_affine(Affine* f, bool* lower, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ val, const double* __restrict__ AL,
                           const double* __restrict__ AU, const uint8_t* __restrict__ keep_col, int row, int col,
                           int max_row_nnz, double zero_tol) {
  const offset_t first = ptr[row], last = ptr[row + 1];
  int live = 0;
  for (offset_t q = first; q < last; ++q)
    if (keep_col[idx[q]] && ++live > max_row_nnz) return false;
  if (live < 2 || live > max_row_nnz || live > kMaxCertifiedRowNnz) return false;
  int pivots = 0;
  double pivot = 0.0;
  for (offset_t q = first; q < last; ++q)
    if (keep_col[idx[q]] && idx[q] == col) { ++pivots; pivot = val[q]; }
  if (pivots != 1) return false;
  double bound = 0.0;
  if (!one_sided(AL[row], AU[row], pivot, zero_tol, lower, &bound)) return false;
  f->constant = bound / pivot;
  f->length = 0;
  if (!isfinite(f->constant)) return false;
  for (offset_t q = first; q < last; ++q) {
    if (!keep_col[idx[q]] || idx[q] == col) continue;
    if (!add_term(idx[q], -val[q] / pivot, f->cols, f->coeffs, &f->length, kMaxAffineTerms)) return false;
  }
  return true;
}

// [min, max] of an expression over the column box (all bounds finite).
__device__ bool affine_range(const Affine& f, const double* __restrict__ l, const double* __restrict__ u, double* lo,
                             double* hi) {
  double a = f.constant, b = f.constant;
  for (int k = 0; k < f.length; ++k) {
    const double lk = l[f.cols[k]], uk = u[f.cols[k]], q = f.coeffs[k];
    if (!isfinite(lk) || !isfinite(uk) || lk > uk) return false;
    a += q >= 0.0 ? q * lk : q * uk;
    b += q >= 0.0 ? q * uk : q * lk;
  }
  if (!isfinite(a) || !isfinite(b)) return false;
  *lo = a;
  *hi = b;
  return true;
}

// rhs - lhs at least tol * (1 + max(|lhs|, |rhs|)).
__device__ bool below_with_margin(double lhs, double rhs, double tol) {
  if (!isfinite(lhs) || !isfinite(rhs)) return false;
  return rhs - lhs >= tol * (1.0 + fmax(fabs(lhs), fabs(rhs)));
}

// max over the box of (lower expression - upper expression).
__device__ bool difference_max(const Affine& lo_f, const Affine& up_f, const double* __restrict__ l,
                               const double* __restrict__ u, double* result) {
  int32_t cols[kMaxDifferenceTerms];
  double coeffs[kMaxDifferenceTerms];
  int length = 0;
  for (int k = 0; k < lo_f.length; ++k)
    if (!add_term(lo_f.cols[k], lo_f.coeffs[k], cols, coeffs, &length, kMaxDifferenceTerms)) return false;
  for (int k = 0; k < up_f.length; ++k)
    if (!add_term(up_f.cols[k], -up_f.coeffs[k], cols, coeffs, &length, kMaxDifferenceTerms)) return false;
  double v = lo_f.constant - up_f.constant;
  for (int k = 0; k < length; ++k) {
    const double lk = l[cols[k]], uk = u[cols[k]];
    if (!isfinite(lk) || !isfinite(uk) || lk > uk) return false;
    v += coeffs[k] >= 0.0 ? coeffs[k] * uk : coeffs[k] * lk;
  }
  if (!isfinite(v)) return false;
  *result = v;
  return true;
}

// The K live rows of column `col` into incident[K*col ..], or false.
template <int K>
__device__ bool live_rows(const offset_t* __restrict__ at_ptr, const int32_t* __restrict__ at_idx,
                          const uint8_t* __restrict__ keep_row, int col, int32_t* __restrict__ incident) {
  int size = 0;
  for (offset_t q = at_ptr[col]; q < at_ptr[col + 1]; ++q) {
    if (!keep_row[at_idx[q]]) continue;
    if (size == K) return false;
    incident[size_t(col) * K + size++] = at_idx[q];
  }
  return size == K;
}

struct ProjectionInput {
  const offset_t *a_ptr, *at_ptr;
  const int32_t *a_idx, *at_idx;
  const double *a_val, *c, *AL, *AU, *l, *u;
  const uint8_t *keep_row, *keep_col;
};

__global__ void tr_detect(int n, ProjectionInput in, int max_row_nnz, double zero_tol, double safety_tol,
                          uint8_t* __restrict__ candidate, int32_t* __restrict__ incident,
                          int32_t* __restrict__ live_count) {
  const int stride = gridDim.x * blockDim.x;
  const int top = (n + stride - 1) / stride * stride;
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < top; col += stride) {
    bool live = false, take = false;
    if (col < n) {
      live = in.keep_col[col] != 0;
      take = live && in.c[col] == 0.0 && isfinite(in.l[col]) && isfinite(in.u[col]) &&
             below_with_margin(in.l[col], in.u[col], safety_tol) &&
             live_rows<2>(in.at_ptr, in.at_idx, in.keep_row, col, incident);
      if (take) {
        const int r0 = incident[size_t(col) * 2], r1 = incident[size_t(col) * 2 + 1];
        Affine f0, f1;
        bool lower0 = false, lower1 = false;
        take = r0 != r1 &&
               row_affine(&f0, &lower0, in.a_ptr, in.a_idx, in.a_val, in.AL, in.AU, in.keep_col, r0, col,
                          max_row_nnz, zero_tol) &&
               row_affine(&f1, &lower1, in.a_ptr, in.a_idx, in.a_val, in.AL, in.AU, in.keep_col, r1, col,
                          max_row_nnz, zero_tol) &&
               lower0 != lower1;
        if (take) {
          const Affine& lo_f = lower0 ? f0 : f1;
          const Affine& up_f = lower0 ? f1 : f0;
          double lo_min, lo_max, up_min, up_max, diff;
          take = affine_range(lo_f, in.l, in.u, &lo_min, &lo_max) && affine_range(up_f, in.l, in.u, &up_min, &up_max) &&
                 below_with_margin(lo_max, in.u[col], safety_tol) &&
                 below_with_margin(in.l[col], up_min, safety_tol) && difference_max(lo_f, up_f, in.l, in.u, &diff) &&
                 below_with_margin(diff, 0.0, safety_tol);
        }
      }
      candidate[col] = take ? 1 : 0;
    }
    block_append(live_count, live);
  }
}

// The McCormick row patterns: z >= x + y - 1 (lower, three entries, side
// -pivot) and z <= x (upper, two entries, side 0), every endpoint entry
// -pivot.
struct McCormickRow {
  bool valid, lower;
  int32_t e0, e1;
};

__device__ McCormickRow mccormick_row(const ProjectionInput& in, int row, int z) {
  McCormickRow r{false, false, -1, -1};
  const offset_t first = in.a_ptr[row], last = in.a_ptr[row + 1];
  int live = 0;
  for (offset_t q = first; q < last; ++q)
    if (in.keep_col[in.a_idx[q]] && ++live > 3) return r;
  if (live != 2 && live != 3) return r;
  double pivot = 0.0;
  int pivots = 0;
  for (offset_t q = first; q < last; ++q)
    if (in.keep_col[in.a_idx[q]] && in.a_idx[q] == z) { pivot = in.a_val[q]; ++pivots; }
  if (pivots != 1 || !isfinite(pivot) || pivot == 0.0) return r;
  double bound;
  const double al = in.AL[row], au = in.AU[row];
  if (isfinite(al) && pos_inf(au)) { r.lower = pivot > 0.0; bound = al; }
  else if (neg_inf(al) && isfinite(au)) { r.lower = pivot < 0.0; bound = au; }
  else return r;
  if (live != (r.lower ? 3 : 2) || bound != (r.lower ? -pivot : 0.0)) return r;
  int ends = 0;
  for (offset_t q = first; q < last; ++q) {
    const int32_t j = in.a_idx[q];
    if (!in.keep_col[j] || j == z) continue;
    if (in.a_val[q] != -pivot || ends >= 2) return r;
    if (ends == 0) r.e0 = j; else r.e1 = j;
    ++ends;
  }
  if (ends != (r.lower ? 2 : 1) || (r.lower && r.e0 == r.e1)) return r;
  r.valid = true;
  return r;
}

__global__ void zc_detect(int n, ProjectionInput in, uint8_t* __restrict__ candidate, int32_t* __restrict__ end0,
                          int32_t* __restrict__ end1, int32_t* __restrict__ incident,
                          int32_t* __restrict__ live_count) {
  const int stride = gridDim.x * blockDim.x;
  const int top = (n + stride - 1) / stride * stride;
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < top; z += stride) {
    bool live = false, take = false;
    if (z < n) {
      live = in.keep_col[z] != 0;
      int32_t x = -1, y = -1;
      if (live && in.c[z] == 0.0 && in.l[z] == 0.0 && in.u[z] == 1.0 &&
          live_rows<3>(in.at_ptr, in.at_idx, in.keep_row, z, incident)) {
        const int32_t* rows = incident + size_t(z) * 3;
        if (rows[0] != rows[1] && rows[0] != rows[2] && rows[1] != rows[2]) {
          const McCormickRow pat[3] = {mccormick_row(in, rows[0], z), mccormick_row(in, rows[1], z),
                                       mccormick_row(in, rows[2], z)};
          int lower_at = -1, ups[2] = {-1, -1}, nup = 0;
          bool ok = true;
          for (int k = 0; k < 3 && ok; ++k) {
            if (!pat[k].valid) ok = false;
            else if (pat[k].lower) { if (lower_at >= 0) ok = false; else lower_at = k; }
            else { if (nup >= 2) ok = false; else ups[nup++] = k; }
          }
          if (ok && lower_at >= 0 && nup == 2) {
            x = pat[lower_at].e0;
            y = pat[lower_at].e1;
            const int32_t ux = pat[ups[0]].e0, uy = pat[ups[1]].e0;
            take = x >= 0 && y >= 0 && x != y && ((ux == x && uy == y) || (ux == y && uy == x)) &&
                   in.l[x] == 0.0 && in.u[x] == 1.0 && in.l[y] == 0.0 && in.u[y] == 1.0;
          }
        }
      }
      candidate[z] = take ? 1 : 0;
      end0[z] = take ? x : -1;
      end1[z] = take ? y : -1;
    }
    block_append(live_count, live);
  }
}

template <int K>
__global__ void count_candidate_rows(int n, const uint8_t* __restrict__ candidate, const int32_t* __restrict__ incident,
                                     int32_t* __restrict__ row_count) {
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n; col += gridDim.x * blockDim.x)
    if (candidate[col])
      for (int k = 0; k < K; ++k) atomicAdd(row_count + incident[size_t(col) * K + k], 1);
}

// A candidate whose rows no other candidate uses (and, for products, whose
// endpoints are not candidates) is selected.
template <int K>
__global__ void select_candidates(int n, const uint8_t* __restrict__ candidate, const int32_t* __restrict__ end0,
                                  const int32_t* __restrict__ end1, const int32_t* __restrict__ incident,
                                  const int32_t* __restrict__ row_count, uint8_t* __restrict__ selected,
                                  int32_t* __restrict__ selected_count) {
  const int stride = gridDim.x * blockDim.x;
  const int top = (n + stride - 1) / stride * stride;
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < top; col += stride) {
    bool take = false;
    if (col < n) {
      take = candidate[col] != 0;
      for (int k = 0; k < K && take; ++k) take = row_count[incident[size_t(col) * K + k]] == 1;
      if (take && end0) take = !candidate[end0[col]] && !candidate[end1[col]];
      selected[col] = take ? 1 : 0;
    }
    block_append(selected_count, take);
  }
}

// The first incident row that bounds the column from below: its pivot and
// finite side (the lower expression of the projected-column record).
template <int K>
__device__ int lower_row(const ProjectionInput& in, const int32_t* __restrict__ incident, int col, double* pivot,
                         double* bound) {
  for (int k = 0; k < K; ++k) {
    const int row = incident[size_t(col) * K + k];
    double v = 0.0;
    int seen = 0;
    for (offset_t q = in.a_ptr[row]; q < in.a_ptr[row + 1]; ++q)
      if (in.a_idx[q] == col) { v = in.a_val[q]; ++seen; }
    if (seen != 1 || !isfinite(v) || v == 0.0) return -1;
    const double al = in.AL[row], au = in.AU[row];
    const bool lo = isfinite(al) && pos_inf(au) && v > 0.0;
    const bool up = neg_inf(al) && isfinite(au) && v < 0.0;
    if (lo || up) {
      *pivot = v;
      *bound = lo ? al : au;
      return row;
    }
  }
  return -1;
}

template <int K>
__global__ void projection_sizes(int n, ProjectionInput in, const uint8_t* __restrict__ selected,
                                 const int32_t* __restrict__ incident, int64_t* __restrict__ records,
                                 int64_t* __restrict__ support, int32_t* __restrict__ failure) {
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n; col += gridDim.x * blockDim.x) {
    records[col] = selected[col] ? 1 : 0;
    int64_t len = 0;
    if (selected[col]) {
      double pivot, bound;
      const int row = lower_row<K>(in, incident, col, &pivot, &bound);
      if (row < 0) {
        atomicOr(failure, 1);
      } else {
        for (offset_t q = in.a_ptr[row]; q < in.a_ptr[row + 1]; ++q)
          len += in.a_idx[q] != col && in.keep_col[in.a_idx[q]];
        if (K == 3 && len != 2) atomicOr(failure, 1);
      }
    }
    support[col] = len;
  }
}

// Record: indices [K, col, rows[K], len, 2, (1, 0), (1, len), support[len]],
// values [box lower (two-row) or 0, side / pivot, -a / pivot ...].
template <int K>
__global__ void projection_pack(int n, ProjectionInput in, const uint8_t* __restrict__ selected,
                                const int32_t* __restrict__ incident, const int64_t* __restrict__ rpos,
                                const int64_t* __restrict__ spos, int32_t* __restrict__ types,
                                int64_t* __restrict__ is, int64_t* __restrict__ vs, int32_t* __restrict__ idx,
                                double* __restrict__ val) {
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n; col += gridDim.x * blockDim.x) {
    if (!selected[col]) continue;
    const int64_t k = rpos[col], s0 = spos[col], len = spos[col + 1] - s0;
    const int64_t ip = int64_t(K + 8) * k + s0, vp = 2 * k + s0;
    types[k] = kFmeCol;
    if (k == 0) { is[0] = 0; vs[0] = 0; }
    is[k + 1] = ip + K + 8 + len;
    vs[k + 1] = vp + 2 + len;
    idx[ip] = K;
    idx[ip + 1] = col;
    for (int j = 0; j < K; ++j) idx[ip + 2 + j] = incident[size_t(col) * K + j];
    idx[ip + 2 + K] = int32_t(len);
    idx[ip + 3 + K] = 2;
    idx[ip + 4 + K] = 1;
    idx[ip + 5 + K] = 0;
    idx[ip + 6 + K] = 1;
    idx[ip + 7 + K] = int32_t(len);
    double pivot = 0.0, bound = 0.0;
    const int row = lower_row<K>(in, incident, col, &pivot, &bound);
    val[vp] = K == 2 ? in.l[col] : 0.0;
    val[vp + 1] = bound / pivot;
    int j = 0;
    for (offset_t q = in.a_ptr[row]; q < in.a_ptr[row + 1]; ++q)
      if (in.a_idx[q] != col && in.keep_col[in.a_idx[q]]) {
        idx[ip + K + 8 + j] = in.a_idx[q];
        val[vp + 2 + j] = -in.a_val[q] / pivot;
        ++j;
      }
  }
}

template <int K>
__global__ void projection_apply(int n, const uint8_t* __restrict__ selected, const int32_t* __restrict__ incident,
                                 uint8_t* __restrict__ keep_row, uint8_t* __restrict__ keep_col) {
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n; col += gridDim.x * blockDim.x)
    if (selected[col]) {
      keep_col[col] = 0;
      for (int k = 0; k < K; ++k) keep_row[incident[size_t(col) * K + k]] = 0;
    }
}

ProjectionInput projection_input(const Plan& plan, const WorkingLp& lp) {
  return ProjectionInput{lp.A.ptr, lp.AT.ptr, lp.A.idx, lp.AT.idx, lp.A.val, plan.c.p, plan.AL.p, plan.AU.p,
                         plan.l.p, plan.u.p, plan.keep_row.p, plan.keep_col.p};
}

// Selection counts, threshold, then the records (before the masks change,
// as the reference builds them) and the deletions.
template <int K>
void commit_projection(Plan& plan, const WorkingLp& lp, const gpp_params& p, const ProjectionInput& in,
                       const uint8_t* candidate, const int32_t* end0, const int32_t* end1, const int32_t* incident,
                       Status& st, int min_candidates, double min_ratio) {
  const int m = lp.m(), n = lp.n();
  auto s = ctx().stream;
  DBuf<int32_t> row_count(size_t(m), s);
  check(cudaMemsetAsync(row_count.p, 0, sizeof(int32_t) * size_t(m), s), "projection row counts");
  DBuf<uint8_t> selected(size_t(n), s);
  GPP_LAUNCH(count_candidate_rows<K>, grid_stride_blocks(n), kThreads, 0, s, n, candidate, incident, row_count.p);
  GPP_LAUNCH(select_candidates<K>, grid_stride_blocks(n), kThreads, 0, s, n, candidate, end0, end1, incident,
             row_count.p, selected.p, st.d);
  const int32_t* counts = st.read(2);
  const int32_t chosen = counts[0], live = counts[1];
  const double ratio = double(chosen) / double(std::max(1, live));
  if (chosen < std::max(1, min_candidates) || !(ratio + 1.0e-15 >= min_ratio)) return;
  if (p.record_postsolve_tape) {
    DBuf<int64_t> rc(size_t(n) + 1, s), sc(size_t(n) + 1, s), rpos(size_t(n) + 1, s), spos(size_t(n) + 1, s);
    st.clear(1);
    GPP_LAUNCH(projection_sizes<K>, grid_stride_blocks(n), kThreads, 0, s, n, in, selected.p, incident, rc.p, sc.p,
               st.d);
    exclusive_scan_i64(rc.p, rpos.p, n, s);
    exclusive_scan_i64(sc.p, spos.p, n, s);
    if (st.read(1)[0]) throw std::runtime_error("projection tape certificate changed before commit");
    const auto [recs, support] = read_scalars(rpos.p + n, spos.p + n);
    if (recs) {
      PostsolveSegment seg = make_segment(recs, int64_t(K + 8) * recs + support, 2 * recs + support);
      GPP_LAUNCH(projection_pack<K>, grid_stride_blocks(n), kThreads, 0, s, n, in, selected.p, incident, rpos.p,
                 spos.p, seg.types.p, seg.is.p, seg.vs.p, seg.idx.p, seg.val.p);
      plan.tape.push_back(std::move(seg));
    }
  }
  GPP_LAUNCH(projection_apply<K>, grid_stride_blocks(n), kThreads, 0, s, n, selected.p, incident, plan.keep_row.p,
             plan.keep_col.p);
  plan.has_change = plan.has_row_action = plan.has_col_action = true;
}

}  // namespace

void rule_two_row_variable_elimination(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  // analyze_two_row_variable_elimination (rule_two_row_variable_elimination.cu:498-612) and
  // build_two_row_variable_elimination_plan (:614-638).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (m <= 0 || n <= 0 || lp.A.nnz <= 0) return;
  const int max_row_nnz = std::max(2, std::min(kMaxCertifiedRowNnz, p.two_row_variable_elimination_max_row_nnz));
  const double safety_tol = std::max(p.two_row_variable_elimination_safety_tol,
                                     std::max(10.0 * p.feasibility_tol, 100.0 * p.zero_tol));
  auto s = ctx().stream;
  const ProjectionInput in = projection_input(plan, lp);
  DBuf<uint8_t> candidate(size_t(n), s);
  DBuf<int32_t> incident(2 * size_t(n), s);
  Status st;
  st.clear(2);
  GPP_LAUNCH(tr_detect, grid_stride_blocks(n), kThreads, 0, s, n, in, max_row_nnz, p.zero_tol, safety_tol,
             candidate.p, incident.p, st.d + 1);
  commit_projection<2>(plan, lp, p, in, candidate.p, nullptr, nullptr, incident.p, st,
                       p.two_row_variable_elimination_min_candidates,
                       p.two_row_variable_elimination_min_candidate_ratio);
}

void rule_zero_cost_product_variables(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  // analyze_zero_cost_product_variables (rule_zero_cost_product_variables.cu:420-544) and
  // build_zero_cost_product_variables_plan (:546-565).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (m <= 0 || n <= 0 || lp.A.nnz <= 0) return;
  auto s = ctx().stream;
  const ProjectionInput in = projection_input(plan, lp);
  DBuf<uint8_t> candidate(size_t(n), s);
  DBuf<int32_t> end0(size_t(n), s), end1(size_t(n), s), incident(3 * size_t(n), s);
  Status st;
  st.clear(2);
  GPP_LAUNCH(zc_detect, grid_stride_blocks(n), kThreads, 0, s, n, in, candidate.p, end0.p, end1.p, incident.p,
             st.d + 1);
  commit_projection<3>(plan, lp, p, in, candidate.p, end0.p, end1.p, incident.p, st,
                       p.zero_cost_product_variables_min_candidates,
                       p.zero_cost_product_variables_min_candidate_ratio);
}

void rule_column_domination(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  const offset_t nnz = lp.A.nnz;
  if (m <= 0 || nnz <= 0 || n < std::max(1, p.column_domination_min_fixed_cols)) return;
  auto s = ctx().stream;
  Status st;
  st.clear(2);
  GPP_LAUNCH(cd_validate_sides, grid_stride_blocks(std::max(m, n)), kThreads, 0, s, m, n, plan.c.p, plan.AL.p,
             plan.AU.p, plan.l.p, plan.u.p, st.d);
  if (st.read(1)[0] != 0) return;
  GPP_LAUNCH(cd_validate_entries, grid_stride_blocks(std::max<int64_t>(nnz, m)), kThreads, 0, s, m, nnz, lp.A.ptr,
             lp.A.idx, lp.A.val, lp.AT.val, plan.c.p, st.d);
  if (st.read(1)[0] != 0) return;
  DBuf<uint8_t> dominated(size_t(n), s);
  GPP_LAUNCH(cd_mark, grid_stride_blocks(n), kThreads, 0, s, n, lp.AT.ptr, plan.c.p, dominated.p, st.d + 1);
  const int32_t candidates = st.read(2)[1];
  const double ratio = double(candidates) / double(n);
  if (candidates < std::max(1, p.column_domination_min_fixed_cols) ||
      ratio + 1.0e-15 < p.column_domination_min_candidate_ratio)
    return;
  GPP_LAUNCH(cd_apply, grid_stride_blocks(n), kThreads, 0, s, n, dominated.p, plan.keep_col.p, plan.l.p, plan.u.p);
  plan.has_col_action = plan.has_change = true;
}

}  // namespace gpp
