// Structure-specific Startup rule: piecewise-linear reformulation of
// variable pairs (reference rules/rule_piecewise_linear_reformulation_variable_pair.cu
// and rules/piecewise_linear_reformulation_variable_pair/{epigraph,shifted_antipodal}.cu).
//
// Both variants see the first 2P columns as P pairs (p_i = column i, m_i =
// column P + i) that the model only uses through the difference p_i - m_i:
// every row holds k pair terms as  v p_i ... - v m_i ...  (plus columns first).
// A merge row  v (p_a - m_a) - v (p_b - m_b) = 0  forces two pairs' differences
// equal; the pairs joined by merge rows (union-find, each component's root its
// smallest pair) collapse to their root's pair, the merge rows go and every
// other row is rewritten on the roots (coefficients of one root summed, zero
// terms dropped).  Primal recovery sets every member's p and m from its
// root's (plus a per-pair shift).
//  * Epigraph (P pairs, then a short positive-cost tail T): each pair has one
//    row  -a p_i - a m_i + b T_j >= L  (its epigraph row).  Pairs have zero
//    cost.  A component keeps one epigraph row, its root's, scaled by
//    sqrt(component size); an equality quotient row is normalised by its
//    first coefficient.  A root column whose component bound leaves no room
//    above its lower bound is removed (fixed).
//  * Shifted antipodal (no tail, 2P columns): c_p = c_m = rho_i > 0; every
//    pair is shifted to its lower bounds (x = l + y), the component keeps the
//    sum of its rho as cost and the smallest widths u - l as bounds; rows
//    subtract the shift sum_k v_k (l_p - l_m) from their sides; the objective
//    constant gains sum_i rho_i (l_p + l_m).
// The epigraph is tried first; when it does not apply the shifted antipodal
// is (rule_..._variable_pair.cu:10-37).  Cheap sampled probes gate both, as in
// the reference: they decide which models are attempted, so they are
// repeated exactly (same sample positions and tests).
// Order-dependent sums: the reference adds a component's rho with atomicAdd
// and the objective constant with cub's device reduction; here both are
// summed in ascending pair order (the same value whenever a component's
// costs are equal, as in the generated models; within rounding otherwise).
#include <algorithm>
#include <cmath>
#include <tuple>

#include "engine.cuh"
#include "sort.hpp"

namespace gpp {

namespace {

constexpr int kMaxQuotientTerms = 6;       // MAX_QUOTIENT_TERMS
constexpr int kEpiMaxProbeDegree = 128;    // epigraph MAX_PROBE_COLUMN_DEGREE
constexpr int kAntiMaxProbeDegree = 64;    // shifted antipodal MAX_PROBE_COLUMN_DEGREE
constexpr int kMaxProbeRows = 1024;        // MAX_PROBE_ROWS
constexpr int kMinProbeMergePercent = 5;   // MIN_PROBE_MERGE_PERCENT
constexpr unsigned long long kNoEdge = ~0ULL;

__device__ __forceinline__ bool valid_row_bounds(double lo, double hi) {
  return !isnan(lo) && !isnan(hi) && lo <= hi && lo != INFINITY && hi != -INFINITY;
}
// epigraph.cu valid_pair_bounds
__device__ __forceinline__ bool epi_pair_bounds(double lo, double hi) {
  return isfinite(lo) && !isnan(hi) && hi >= lo && (!isfinite(hi) || isfinite(hi - lo));
}
// shifted_antipodal.cu _valid_shifted_pair_bounds (+ the finite-width test)
__device__ __forceinline__ bool anti_pair_bounds(double lo, double hi) {
  return isfinite(lo) && !isnan(hi) && hi >= lo && (!isfinite(hi) || isfinite(hi - lo));
}

// A row that merges pairs a and b:  v p_a - v p_b - v m_a + v m_b = 0.
__device__ bool merge_row_shape(offset_t lo, offset_t len, const int32_t* idx, const double* val, double al, double au,
                                int P) {
  if (len != 4 || al != 0.0 || au != 0.0) return false;
  const int32_t a = idx[lo], b = idx[lo + 1];
  const double va = val[lo], vb = val[lo + 1];
  return a >= 0 && a < P && b >= 0 && b < P && a != b && idx[lo + 2] == a + P && idx[lo + 3] == b + P &&
         isfinite(va) && isfinite(vb) && va != 0.0 && va == -vb && va == -val[lo + 2] && vb == -val[lo + 3];
}

// Share of sampled rows (row = s * rows / probes) that are merge rows
// (kernel_quick_..._edge_probe / _kernel_quick_merge_row_probe).
__global__ void merge_row_probe(int rows, int P, int probes, const offset_t* __restrict__ ptr,
                                const int32_t* __restrict__ idx, const double* __restrict__ val,
                                const double* __restrict__ AL, const double* __restrict__ AU,
                                int32_t* __restrict__ count) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < probes; s += gridDim.x * blockDim.x) {
    const int row = int(int64_t(s) * rows / probes);
    const offset_t lo = ptr[row];
    if (merge_row_shape(lo, ptr[row + 1] - lo, idx, val, AL[row], AU[row], P)) atomicAdd(count, 1);
  }
}

// Sampled pairs (pair = s * P / probes): epigraph version
// (kernel_quick_..._epigraph_pair_probe).
__global__ void epi_pair_probe(int P, int cols, int probes, const offset_t* __restrict__ at_ptr,
                               const int32_t* __restrict__ at_idx, const double* __restrict__ at_val,
                               const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                               const double* __restrict__ val, const double* __restrict__ AL,
                               const double* __restrict__ AU, const double* __restrict__ c,
                               const double* __restrict__ l, const double* __restrict__ u, int32_t* __restrict__ failed) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < probes; s += gridDim.x * blockDim.x) {
    const int pair = int(int64_t(s) * P / probes), mate = pair + P;
    const offset_t b = at_ptr[pair], mb = at_ptr[mate];
    const int degree = at_ptr[pair + 1] - b;
    bool ok = degree >= 2 && degree <= kEpiMaxProbeDegree && degree == at_ptr[mate + 1] - mb && c[pair] == 0.0 &&
              c[mate] == 0.0 && epi_pair_bounds(l[pair], u[pair]) && epi_pair_bounds(l[mate], u[mate]);
    int same = 0;
    if (ok) {
      for (int k = 0; k < degree; ++k) {
        const int32_t row = at_idx[b + k];
        const double v = at_val[b + k], mv = at_val[mb + k];
        if (row != at_idx[mb + k] || !isfinite(v) || !isfinite(mv) || v == 0.0) { ok = false; break; }
        if (v == mv) {
          ++same;
          const offset_t rb = ptr[row];
          ok = ptr[row + 1] - rb == 3 && idx[rb] == pair && idx[rb + 1] == mate && idx[rb + 2] >= 2 * P &&
               idx[rb + 2] < cols && val[rb] == val[rb + 1] && val[rb] < 0.0 && isfinite(val[rb + 2]) &&
               val[rb + 2] > 0.0 && isfinite(AL[row]) && AU[row] == INFINITY;
          if (!ok) break;
        } else if (v != -mv) {
          ok = false;
          break;
        }
      }
    }
    if (!ok || same != 1) atomicExch(failed, 1);
  }
}

// Sampled pairs: shifted antipodal version (_kernel_quick_..._shifted_antipodal_probe).
__global__ void anti_pair_probe(int P, int probes, const offset_t* __restrict__ at_ptr,
                                const int32_t* __restrict__ at_idx, const double* __restrict__ at_val,
                                const double* __restrict__ c, const double* __restrict__ l,
                                const double* __restrict__ u, int32_t* __restrict__ failed) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < probes; s += gridDim.x * blockDim.x) {
    const int col = int(int64_t(s) * P / probes), mate = col + P;
    const offset_t b = at_ptr[col], e = at_ptr[col + 1], mb = at_ptr[mate];
    const int degree = e - b;
    bool ok = degree >= 1 && degree <= kAntiMaxProbeDegree && degree == at_ptr[mate + 1] - mb;
    ok = ok && isfinite(c[col]) && c[col] > 0.0 && c[col] == c[mate];
    ok = ok && anti_pair_bounds(l[col], u[col]) && anti_pair_bounds(l[mate], u[mate]);
    if (ok)
      for (int k = 0; k < degree; ++k)
        if (at_idx[b + k] != at_idx[mb + k] || at_val[b + k] != -at_val[mb + k]) { ok = false; break; }
    if (!ok) atomicExch(failed, 1);
  }
}

// ---- union-find over the merge edges (roots are the smallest pair) -----------------------

__global__ void uf_init(int P, int32_t* __restrict__ parent) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) parent[i] = i;
}
__device__ int32_t uf_find(int32_t* parent, int32_t v) {
  int32_t cur = v;
  for (;;) {
    const int32_t next = *(volatile int32_t*)(parent + cur);
    const int32_t grand = *(volatile int32_t*)(parent + next);
    if (next == grand) {
      if (cur != next) atomicCAS(parent + cur, next, grand);
      return next;
    }
    atomicCAS(parent + cur, next, grand);
    cur = grand;
  }
}
// Links point from a larger root to a smaller one, so the forest stays
// acyclic and every retry makes progress.
__global__ void uf_union(int rows, const unsigned long long* __restrict__ edge, int32_t* parent) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const unsigned long long e = edge[r];
    if (e == kNoEdge) continue;
    const int32_t a = int32_t(e >> 32), b = int32_t(e & 0xffffffffu);
    for (;;) {
      const int32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
      if (ra == rb) break;
      const int32_t hi = max(ra, rb), lo = min(ra, rb);
      if (atomicCAS(parent + hi, hi, lo) == hi) break;
    }
  }
}
// Every pair points at its root; roots[0] counts the roots (one atomic per
// warp).
__global__ void uf_flatten(int P, int32_t* parent, int32_t* __restrict__ roots) {
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < P; base += stride) {
    const int i = base + threadIdx.x;
    bool root = false;
    if (i < P) {
      const int32_t r = uf_find(parent, i);
      parent[i] = r;
      root = r == i;
    }
    const unsigned b = __ballot_sync(0xffffffffu, root);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(roots, __popc(b));
  }
}
__global__ void fill_minus_one(int32_t* p, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = -1;
}

// Per component, in ascending pair order (pairs sorted by (root, pair)):
// size, the min of two per-pair values, and the sum of a third.
__global__ void component_keys(int P, const int32_t* __restrict__ parent, uint64_t* __restrict__ keys,
                               int32_t* __restrict__ vals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
    keys[i] = (uint64_t(uint32_t(parent[i])) << 32) | uint32_t(i);
    vals[i] = i;
  }
}
// min that ignores NaN operands, as the reference's CAS loop (`value < old`)
// does, starting from +inf.
__device__ __forceinline__ double min_keep(double acc, double v) { return v < acc ? v : acc; }

// ---- quotient rows (collect_..._quotient_row / _collect_quotient_row) -----------------------

// Roots and coefficients of a row's pair terms, sorted by root (stable
// insertion sort), equal roots summed, zeros dropped; the shift sum_k v_k
// shift_k in row order.  Returns the number of terms left, or -1 when a
// value is not finite.
__device__ int quotient_row(offset_t lo, int terms, const int32_t* __restrict__ idx, const double* __restrict__ val,
                            const int32_t* __restrict__ parent, const double* __restrict__ pair_shift,
                            int32_t* roots, double* coef, double* shift) {
  *shift = 0.0;
  for (int k = 0; k < terms; ++k) {
    const int32_t pair = idx[lo + k];
    roots[k] = parent[pair];
    coef[k] = val[lo + k];
    const double t = coef[k] * pair_shift[pair];
    if (!isfinite(coef[k]) || !isfinite(t)) return -1;
    *shift += t;
    if (!isfinite(*shift)) return -1;
  }
  for (int i = 1; i < terms; ++i) {
    const int32_t r = roots[i];
    const double v = coef[i];
    int j = i;
    while (j > 0 && roots[j - 1] > r) {
      roots[j] = roots[j - 1];
      coef[j] = coef[j - 1];
      --j;
    }
    roots[j] = r;
    coef[j] = v;
  }
  int merged = 0;
  for (int i = 0; i < terms; ++i) {
    if (merged > 0 && roots[merged - 1] == roots[i]) {
      coef[merged - 1] += coef[i];
      if (!isfinite(coef[merged - 1])) return -1;
    } else {
      roots[merged] = roots[i];
      coef[merged] = coef[i];
      ++merged;
    }
  }
  int active = 0;
  for (int i = 0; i < merged; ++i)
    if (coef[i] != 0.0) {
      roots[active] = roots[i];
      coef[active] = coef[i];
      ++active;
    }
  return active;
}

// Every non-epigraph row: k pair terms, plus columns first, minus columns
// mirrored with negated values.  Returns the term count or 0 when the row
// does not have that shape.
__device__ int pair_terms(offset_t lo, offset_t len, const int32_t* __restrict__ idx, const double* __restrict__ val,
                          int P, int max_terms, bool anti) {
  if (len < 2 || (len & 1)) return 0;
  const int terms = int(len / 2);
  if (terms < 1 || terms > max_terms || terms > kMaxQuotientTerms) return 0;
  for (int k = 0; k < terms; ++k) {
    const int32_t p = idx[lo + k], m = idx[lo + terms + k];
    const double vp = val[lo + k], vm = val[lo + terms + k];
    if (p < 0 || p >= P || m != p + P || !isfinite(vp) || (anti && !isfinite(vm)) || vp == 0.0 || vp != -vm) return 0;
  }
  return terms;
}

// ---- epigraph ----------------------------------------------------------------------------

struct EpiArgs {
  const offset_t* ptr;
  const int32_t* idx;
  const double* val;
  const double *AL, *AU, *c, *l, *u;
  int rows, cols, P, max_terms;
};

// kernel_validate_..._epigraph_columns: zero-cost pairs with finite lower
// bounds, positive-cost tail columns.
__global__ void epi_columns(EpiArgs g, double* __restrict__ shift, double* __restrict__ lower_sum,
                            int32_t* __restrict__ status) {
  const int top = max(g.P, g.cols - 2 * g.P);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < top; i += gridDim.x * blockDim.x) {
    if (i < g.P) {
      const int mate = i + g.P;
      const double lp = g.l[i], ln = g.l[mate];
      bool ok = g.c[i] == 0.0 && g.c[mate] == 0.0 && epi_pair_bounds(lp, g.u[i]) && epi_pair_bounds(ln, g.u[mate]);
      const double sh = lp - ln, sum = lp + ln;
      ok = ok && isfinite(sh) && isfinite(sum);
      shift[i] = ok ? sh : 0.0;
      lower_sum[i] = ok ? sum : 0.0;
      if (!ok) atomicOr(status, 1);
    }
    const int t = 2 * g.P + i;
    if (t < g.cols) {
      const bool ok = isfinite(g.c[t]) && g.c[t] > 0.0 && !isnan(g.l[t]) && !isnan(g.u[t]) && g.l[t] <= g.u[t] &&
                      g.l[t] != INFINITY && g.u[t] != -INFINITY;
      if (!ok) atomicOr(status, 1);
    }
  }
}

// kernel_classify_..._epigraph_rows: epigraph rows claim their pair, merge
// rows become edges, every other row must be a pair-term row.
// counts: [0] edges, [1] epigraph rows.
__global__ void epi_classify(EpiArgs g, const double* __restrict__ shift, unsigned long long* __restrict__ edge,
                             int32_t* __restrict__ g_pair_by_row, int32_t* __restrict__ pair_g_row,
                             int32_t* __restrict__ pair_tail, double* __restrict__ pair_gcoef,
                             int32_t* __restrict__ counts, int32_t* __restrict__ status) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < g.rows; row += gridDim.x * blockDim.x) {
    const offset_t lo = g.ptr[row], len = g.ptr[row + 1] - lo;
    const double al = g.AL[row], au = g.AU[row];
    bool ok = valid_row_bounds(al, au);
    unsigned long long packed = kNoEdge;
    int32_t gp = -1;
    if (ok && len == 3) {
      const int32_t p = g.idx[lo], n = g.idx[lo + 1], t = g.idx[lo + 2];
      const double vp = g.val[lo], vn = g.val[lo + 1], vt = g.val[lo + 2];
      ok = p >= 0 && p < g.P && n == p + g.P && t >= 2 * g.P && t < g.cols && isfinite(vp) && vp < 0.0 && vp == vn &&
           isfinite(vt) && vt > 0.0 && isfinite(al) && au == INFINITY;
      if (ok) {
        if (atomicCAS(pair_g_row + p, -1, row) != -1) {
          ok = false;
        } else {
          pair_tail[p] = t;
          pair_gcoef[p] = vp;
          gp = p;
          atomicAdd(counts + 1, 1);
        }
      }
    } else if (ok) {
      const int terms = pair_terms(lo, len, g.idx, g.val, g.P, g.max_terms, false);
      ok = terms > 0;
      if (ok && terms == 2 && al == 0.0 && au == 0.0 && g.val[lo] == -g.val[lo + 1]) {
        const uint32_t a = uint32_t(g.idx[lo]), b = uint32_t(g.idx[lo + 1]);
        if (a == b || shift[a] != shift[b]) {
          ok = false;
        } else {
          packed = (uint64_t(min(a, b)) << 32) | uint64_t(max(a, b));
          atomicAdd(counts, 1);
        }
      }
    }
    edge[row] = packed;
    g_pair_by_row[row] = gp;
    if (!ok) atomicOr(status, 2);
  }
}

// Component aggregates in pair order: size, min u of the plus and of the
// minus columns (kernel_aggregate_..._epigraph_uppers).
__global__ void epi_aggregate(int P, const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals,
                              const double* __restrict__ u, int32_t* __restrict__ size, double* __restrict__ plus_up,
                              double* __restrict__ minus_up) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P; q += gridDim.x * blockDim.x) {
    const uint32_t r = uint32_t(keys[q] >> 32);
    if (q > 0 && uint32_t(keys[q - 1] >> 32) == r) continue;
    int count = 0;
    double pu = INFINITY, mu = INFINITY;
    for (int k = q; k < P && uint32_t(keys[k] >> 32) == r; ++k) {
      const int pair = vals[k];
      ++count;
      pu = min_keep(pu, u[pair]);
      mu = min_keep(mu, u[pair + P]);
    }
    size[r] = count;
    plus_up[r] = pu;
    minus_up[r] = mu;
  }
}

// kernel_validate_..._epigraph: every pair agrees with its root on shifts,
// lower bounds, tail column and epigraph row; roots have room above l.
__global__ void epi_validate(EpiArgs g, const int32_t* __restrict__ parent, const int32_t* __restrict__ pair_g_row,
                             const int32_t* __restrict__ pair_tail, const double* __restrict__ pair_gcoef,
                             const double* __restrict__ shift, const double* __restrict__ lower_sum,
                             const double* __restrict__ plus_up, const double* __restrict__ minus_up,
                             int32_t* __restrict__ status) {
  for (int pair = blockIdx.x * blockDim.x + threadIdx.x; pair < g.P; pair += gridDim.x * blockDim.x) {
    const int32_t root = parent[pair];
    const int32_t row = pair_g_row[pair];
    const int32_t rrow = root >= 0 && root < g.P ? pair_g_row[root] : -1;
    bool ok = root >= 0 && root < g.P && row >= 0 && rrow >= 0 && shift[pair] == shift[root] &&
              lower_sum[pair] == lower_sum[root] && g.l[pair] == g.l[root] && g.l[pair + g.P] == g.l[root + g.P] &&
              pair_tail[pair] == pair_tail[root] && pair_gcoef[pair] == pair_gcoef[root] &&
              g.AL[row] == g.AL[rrow] && g.AU[row] == g.AU[rrow] && g.val[g.ptr[row] + 2] == g.val[g.ptr[rrow] + 2];
    if (ok && pair == root)
      ok = !isnan(plus_up[root]) && !isnan(minus_up[root]) && plus_up[root] >= g.l[root] &&
           minus_up[root] >= g.l[root + g.P];
    if (!ok) atomicOr(status, 4);
  }
}

// kernel_count_..._epigraph_rewritten_rows: per-row output size, sides and
// keep flag into scratch (committed only when the whole rewrite is valid).
// status: 32 = a row cannot be rewritten exactly, 1 = a row became 0 = b != 0.
struct RowOut {
  int32_t* count;
  uint8_t* keep;
  double *AL, *AU;
};
__global__ void epi_rows(EpiArgs g, const int32_t* __restrict__ parent, const int32_t* __restrict__ size,
                         const double* __restrict__ shift, const unsigned long long* __restrict__ edge,
                         const int32_t* __restrict__ g_pair_by_row, double feas_tol, RowOut out,
                         int32_t* __restrict__ removed, int32_t* __restrict__ status) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < g.rows; row += gridDim.x * blockDim.x) {
    const int32_t pair = g_pair_by_row[row];
    const double al = g.AL[row], au = g.AU[row];
    out.AL[row] = al;
    out.AU[row] = au;
    if (pair >= 0) {
      if (parent[pair] != pair) {
        out.count[row] = 0;
        out.keep[row] = 0;
        atomicAdd(removed, 1);
        continue;
      }
      // The kept epigraph row stands for the component's identical rows;
      // sqrt(size) keeps their weight in the residual 2-norm.
      const double w = sqrt(double(size[pair]));
      const double lo = al * w, hi = isfinite(au) ? au * w : au;
      if (size[pair] <= 0 || !isfinite(w) || !valid_row_bounds(lo, hi) || (isfinite(al) && !isfinite(lo)) ||
          (isfinite(au) && !isfinite(hi))) {
        atomicOr(status, 32);
        out.count[row] = 0;
        out.keep[row] = 1;
      } else {
        out.AL[row] = lo;
        out.AU[row] = hi;
        out.count[row] = 3;
        out.keep[row] = 1;
      }
      continue;
    }
    if (edge[row] != kNoEdge) {
      out.AL[row] = 0.0;
      out.AU[row] = 0.0;
      out.count[row] = 0;
      out.keep[row] = 0;
      atomicAdd(removed, 1);
      continue;
    }
    int32_t roots[kMaxQuotientTerms];
    double coef[kMaxQuotientTerms], sh;
    const offset_t lo = g.ptr[row];
    const int active = quotient_row(lo, int((g.ptr[row + 1] - lo) / 2), g.idx, g.val, parent, shift, roots, coef, &sh);
    if (active < 0) {
      atomicOr(status, 32);
      out.count[row] = 0;
      out.keep[row] = 1;
      continue;
    }
    bool norm_ok = true;
    if (active > 0 && isfinite(al) && al == au) {
      const double scale = coef[0];
      const double rhs = al / scale;
      norm_ok = isfinite(scale) && scale != 0.0 && isfinite(rhs);
      for (int k = 0; k < active && norm_ok; ++k) norm_ok = isfinite(coef[k] / scale);
      if (norm_ok) {
        out.AL[row] = rhs;
        out.AU[row] = rhs;
      }
    }
    if (!norm_ok || !valid_row_bounds(al, au)) {
      atomicOr(status, 32);
      out.AL[row] = al;
      out.AU[row] = au;
      out.count[row] = 0;
      out.keep[row] = 1;
      continue;
    }
    out.count[row] = 2 * active;
    if (active == 0) {
      out.keep[row] = 0;
      atomicAdd(removed, 1);
      if (al > feas_tol || au < -feas_tol) atomicOr(status, 1);
    } else {
      out.keep[row] = 1;
    }
  }
}

// kernel_fill_..._epigraph_rewritten_rows (one thread per row: at most six
// terms per row).
__global__ void epi_fill(EpiArgs g, const int32_t* __restrict__ parent, const int32_t* __restrict__ size,
                         const double* __restrict__ shift, const int32_t* __restrict__ pair_tail,
                         const unsigned long long* __restrict__ edge, const int32_t* __restrict__ g_pair_by_row,
                         const offset_t* __restrict__ optr, int32_t* __restrict__ oidx, double* __restrict__ oval) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < g.rows; row += gridDim.x * blockDim.x) {
    const offset_t w0 = optr[row];
    if (w0 == optr[row + 1]) continue;
    const int32_t pair = g_pair_by_row[row];
    const offset_t lo = g.ptr[row];
    if (pair >= 0) {
      const double w = sqrt(double(size[pair]));
      oidx[w0] = pair;
      oval[w0] = w * g.val[lo];
      oidx[w0 + 1] = pair + g.P;
      oval[w0 + 1] = w * g.val[lo + 1];
      oidx[w0 + 2] = pair_tail[pair];
      oval[w0 + 2] = w * g.val[lo + 2];
      continue;
    }
    if (edge[row] != kNoEdge) continue;
    int32_t roots[kMaxQuotientTerms];
    double coef[kMaxQuotientTerms], sh;
    const int active = quotient_row(lo, int((g.ptr[row + 1] - lo) / 2), g.idx, g.val, parent, shift, roots, coef, &sh);
    if (active <= 0) continue;
    const double scale = isfinite(g.AL[row]) && g.AL[row] == g.AU[row] ? coef[0] : 1.0;
    for (int k = 0; k < active; ++k) {
      oidx[w0 + k] = roots[k];
      oval[w0 + k] = coef[k] / scale;
      oidx[w0 + active + k] = roots[k] + g.P;
      oval[w0 + active + k] = -coef[k] / scale;
    }
  }
}

// kernel_prepare_..._epigraph_columns: roots keep their pair (a column with
// no room above its lower bound goes), members go.
__global__ void epi_columns_apply(int P, const int32_t* __restrict__ parent, const double* __restrict__ plus_up,
                                  const double* __restrict__ minus_up, uint8_t* __restrict__ keep_col,
                                  double* __restrict__ c, double* __restrict__ l, double* __restrict__ u) {
  for (int pair = blockIdx.x * blockDim.x + threadIdx.x; pair < P; pair += gridDim.x * blockDim.x) {
    const bool root = parent[pair] == pair;
    keep_col[pair] = root && plus_up[pair] > l[pair] ? 1 : 0;
    keep_col[pair + P] = root && minus_up[pair] > l[pair + P] ? 1 : 0;
    if (root) {
      c[pair] = 0.0;
      c[pair + P] = 0.0;
      u[pair] = plus_up[pair];
      u[pair + P] = minus_up[pair];
    }
  }
}

// ---- shifted antipodal ---------------------------------------------------------------------

// _kernel_validate_pair_metadata: rho = c_p = c_m > 0, finite widths;
// shift = l_p - l_m, constant = rho (l_p + l_m).
__global__ void anti_columns(int P, const double* __restrict__ c, const double* __restrict__ l,
                             const double* __restrict__ u, double* __restrict__ shift, double* __restrict__ constant,
                             int32_t* __restrict__ status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
    const int mate = i + P;
    const double rho = c[i], lp = l[i], ln = l[mate];
    bool ok = isfinite(rho) && rho > 0.0 && rho == c[mate] && anti_pair_bounds(lp, u[i]) &&
              anti_pair_bounds(ln, u[mate]);
    const double sh = lp - ln, k = rho * (lp + ln);
    ok = ok && isfinite(sh) && isfinite(k);
    shift[i] = ok ? sh : 0.0;
    constant[i] = ok ? k : 0.0;
    if (!ok) atomicOr(status, 1);
  }
}

// _kernel_classify_..._shifted_antipodal_rows.  counts[0]: edges.
__global__ void anti_classify(const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                              const double* __restrict__ val, const double* __restrict__ AL,
                              const double* __restrict__ AU, const double* __restrict__ shift, int rows, int P,
                              int max_terms, unsigned long long* __restrict__ edge, int32_t* __restrict__ counts,
                              int32_t* __restrict__ status) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
    const offset_t lo = ptr[row], len = ptr[row + 1] - lo;
    const double al = AL[row], au = AU[row];
    bool ok = valid_row_bounds(al, au);
    unsigned long long packed = kNoEdge;
    const int terms = ok ? pair_terms(lo, len, idx, val, P, max_terms, true) : 0;
    ok = ok && terms > 0;
    if (ok && terms == 2 && al == 0.0 && au == 0.0 && val[lo] == -val[lo + 1]) {
      const uint32_t a = uint32_t(idx[lo]), b = uint32_t(idx[lo + 1]);
      if (shift[a] != shift[b]) {
        ok = false;
      } else {
        packed = (uint64_t(min(a, b)) << 32) | uint64_t(max(a, b));
        atomicAdd(counts, 1);
      }
    }
    edge[row] = packed;
    if (!ok) atomicOr(status, 1);
  }
}

// Components in pair order: min widths u - l of the plus and minus columns,
// the sum of rho (_kernel_aggregate_component_metadata); invalid roots set
// status 16 (_kernel_validate_component_metadata).
__global__ void anti_aggregate(int P, const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals,
                               const double* __restrict__ c, const double* __restrict__ l,
                               const double* __restrict__ u, double* __restrict__ plus_cap,
                               double* __restrict__ minus_cap, double* __restrict__ rho, int32_t* __restrict__ status) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P; q += gridDim.x * blockDim.x) {
    const uint32_t r = uint32_t(keys[q] >> 32);
    if (q > 0 && uint32_t(keys[q - 1] >> 32) == r) continue;
    double pc = INFINITY, mc = INFINITY, sum = 0.0;
    for (int k = q; k < P && uint32_t(keys[k] >> 32) == r; ++k) {
      const int pair = vals[k];
      pc = min_keep(pc, u[pair] - l[pair]);
      mc = min_keep(mc, u[pair + P] - l[pair + P]);
      sum += c[pair];
    }
    plus_cap[r] = pc;
    minus_cap[r] = mc;
    rho[r] = sum;
    if (isnan(pc) || isnan(mc) || pc < 0.0 || mc < 0.0 || !isfinite(sum) || sum <= 0.0) atomicOr(status, 16);
  }
}

// Every merge edge ended inside one component (_kernel_verify_...).
__global__ void anti_verify(int rows, const unsigned long long* __restrict__ edge, const int32_t* __restrict__ parent,
                            const double* __restrict__ shift, int32_t* __restrict__ status) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const unsigned long long e = edge[r];
    if (e == kNoEdge) continue;
    const int32_t a = int32_t(e >> 32), b = int32_t(e & 0xffffffffu);
    if (parent[a] != parent[b] || shift[a] != shift[b]) atomicOr(status, 8);
  }
}

// _kernel_count_rewritten_rows (shifted antipodal): sides minus the row's
// shift; a row left with no terms goes (infeasible unless 0 within tolerance).
__global__ void anti_rows(const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                          const double* __restrict__ val, const double* __restrict__ AL, const double* __restrict__ AU,
                          int rows, const int32_t* __restrict__ parent, const double* __restrict__ shift,
                          const unsigned long long* __restrict__ edge, double feas_tol, RowOut out,
                          int32_t* __restrict__ removed, int32_t* __restrict__ status) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
    const double al = AL[row], au = AU[row];
    out.AL[row] = al;
    out.AU[row] = au;
    if (edge[row] != kNoEdge) {
      out.AL[row] = 0.0;
      out.AU[row] = 0.0;
      out.count[row] = 0;
      out.keep[row] = 0;
      atomicAdd(removed, 1);
      continue;
    }
    int32_t roots[kMaxQuotientTerms];
    double coef[kMaxQuotientTerms], sh;
    const offset_t lo = ptr[row];
    const int active = quotient_row(lo, int((ptr[row + 1] - lo) / 2), idx, val, parent, shift, roots, coef, &sh);
    if (active < 0) {
      out.count[row] = 0;
      out.keep[row] = 1;
      atomicOr(status, 32);
      continue;
    }
    const double lower = al - sh, upper = au - sh;
    if (!valid_row_bounds(lower, upper) || (isfinite(al) && !isfinite(lower)) || (isfinite(au) && !isfinite(upper))) {
      out.count[row] = 0;
      out.keep[row] = 1;
      atomicOr(status, 32);
      continue;
    }
    out.AL[row] = lower;
    out.AU[row] = upper;
    out.count[row] = 2 * active;
    if (active == 0) {
      out.keep[row] = 0;
      atomicAdd(removed, 1);
      if (lower > feas_tol || upper < -feas_tol) atomicOr(status, 1);
    } else {
      out.keep[row] = 1;
    }
  }
}

__global__ void anti_fill(const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                          const double* __restrict__ val, int rows, int P, const int32_t* __restrict__ parent,
                          const double* __restrict__ shift, const offset_t* __restrict__ optr,
                          int32_t* __restrict__ oidx, double* __restrict__ oval) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
    const offset_t w0 = optr[row];
    if (w0 == optr[row + 1]) continue;
    int32_t roots[kMaxQuotientTerms];
    double coef[kMaxQuotientTerms], sh;
    const offset_t lo = ptr[row];
    const int active = quotient_row(lo, int((ptr[row + 1] - lo) / 2), idx, val, parent, shift, roots, coef, &sh);
    for (int k = 0; k < active; ++k) {
      oidx[w0 + k] = roots[k];
      oval[w0 + k] = coef[k];
      oidx[w0 + active + k] = roots[k] + P;
      oval[w0 + active + k] = -coef[k];
    }
  }
}

// _kernel_prepare_..._shifted_antipodal_columns.
__global__ void anti_columns_apply(int P, const int32_t* __restrict__ parent, const double* __restrict__ plus_cap,
                                   const double* __restrict__ minus_cap, const double* __restrict__ rho,
                                   uint8_t* __restrict__ keep_col, double* __restrict__ c, double* __restrict__ l,
                                   double* __restrict__ u) {
  for (int pair = blockIdx.x * blockDim.x + threadIdx.x; pair < P; pair += gridDim.x * blockDim.x) {
    const bool root = parent[pair] == pair;
    keep_col[pair] = root ? 1 : 0;
    keep_col[pair + P] = root ? 1 : 0;
    if (root) {
      c[pair] = rho[pair];
      c[pair + P] = rho[pair];
      l[pair] = 0.0;
      l[pair + P] = 0.0;
      u[pair] = plus_cap[pair];
      u[pair + P] = minus_cap[pair];
    }
  }
}

// ---- shared commit and recovery ----------------------------------------------------------

__global__ void commit_rows(int rows, const uint8_t* __restrict__ keep, const double* __restrict__ al,
                            const double* __restrict__ au, uint8_t* __restrict__ keep_row, double* __restrict__ AL,
                            double* __restrict__ AU) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    keep_row[r] = keep[r];
    AL[r] = al[r];
    AU[r] = au[r];
  }
}

// capture_variable_pair_recovery_device (device_recovery.cu:655-670).
__global__ void pair_recovery(int P, const int32_t* __restrict__ parent, const double* __restrict__ l, int shifted,
                              int32_t* __restrict__ plus, int32_t* __restrict__ minus, int32_t* __restrict__ root_plus,
                              int32_t* __restrict__ root_minus, double* __restrict__ plus_shift,
                              double* __restrict__ minus_shift) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
    plus[i] = i;
    minus[i] = i + P;
    root_plus[i] = parent[i];
    root_minus[i] = parent[i] + P;
    plus_shift[i] = shifted ? l[i] : 0.0;
    minus_shift[i] = shifted ? l[i + P] : 0.0;
  }
}

std::unique_ptr<VarPairRecovery> make_recovery(int P, const int32_t* parent, const double* l, bool shifted,
                                               cudaStream_t s) {
  auto r = std::make_unique<VarPairRecovery>();
  r->count = P;
  r->plus.alloc(size_t(P), s);
  r->minus.alloc(size_t(P), s);
  r->root_plus.alloc(size_t(P), s);
  r->root_minus.alloc(size_t(P), s);
  r->plus_shift.alloc(size_t(P), s);
  r->minus_shift.alloc(size_t(P), s);
  GPP_LAUNCH(pair_recovery, grid_stride_blocks(P), kThreads, 0, s, P, parent, l, int(shifted), r->plus.p, r->minus.p,
             r->root_plus.p, r->root_minus.p, r->plus_shift.p, r->minus_shift.p);
  return r;
}

// Union-find over the edges, flattened: returns the number of components.
int components(int P, int rows, const unsigned long long* edge, DBuf<int32_t>& parent, cudaStream_t s) {
  parent.alloc(size_t(P), s);
  DBuf<int32_t> roots(1, s);
  roots.zero();
  GPP_LAUNCH(uf_init, grid_stride_blocks(P), kThreads, 0, s, P, parent.p);
  GPP_LAUNCH(uf_union, grid_stride_blocks(rows), kThreads, 0, s, rows, edge, parent.p);
  GPP_LAUNCH(uf_flatten, grid_stride_blocks(P), kThreads, 0, s, P, parent.p, roots.p);
  return read_scalar(roots.p);
}

// The sampled merge-row share: at least 5% of min(rows, 1024) sampled rows.
bool merge_rows_dense_enough(const DevCsr& A, const double* AL, const double* AU, int P, cudaStream_t s,
                             const int32_t* failed_probe, int32_t* counts) {
  const int probes = std::min(A.rows, kMaxProbeRows);
  GPP_LAUNCH(merge_row_probe, grid_stride_blocks(probes), kThreads, 0, s, A.rows, P, probes, A.ptr, A.idx, A.val,
             AL, AU, counts);
  int32_t failed = 0, merges = 0;
  std::tie(failed, merges) = read_scalars(failed_probe, counts);
  return failed == 0 && int64_t(merges) * 100 >= int64_t(probes) * kMinProbeMergePercent;
}

// ---- epigraph -----------------------------------------------------------------------------

// infer_..._epigraph_layout (epigraph.cu:55-121): the objective ends in
// 1..max_tail positive entries preceded by a zero, and what comes before is
// an even number of pair columns, at least min_pairs pairs.
bool epigraph_layout(const WorkingLp& lp, const gpp_params& p, int* pairs) {
  const int cols = lp.n();
  if (cols <= 2 || !lp.c) return false;
  const int min_pairs = std::max(1, p.piecewise_linear_reformulation_variable_pair_epigraph_min_pairs);
  if (cols < 2LL * min_pairs + 1 || lp.m() < 2LL * min_pairs || lp.A.nnz < 7LL * min_pairs) return false;
  const int max_tail = std::max(1, std::min(p.piecewise_linear_reformulation_variable_pair_epigraph_max_tail_cols, 8));
  const int copy = std::min(cols, max_tail + 1);
  double suffix[9] = {};
  check(cudaMemcpyAsync(suffix, lp.c + (cols - copy), sizeof(double) * size_t(copy), cudaMemcpyDeviceToHost,
                        ctx().stream),
        "epigraph objective suffix");
  ctx().sync("epigraph layout");
  const double last = suffix[copy - 1];
  if (!std::isfinite(last) || last <= 0.0) return false;
  int tail = 0;
  for (int k = copy - 1; k >= 0; --k) {
    if (std::isfinite(suffix[k]) && suffix[k] > 0.0 && tail < max_tail) { ++tail; continue; }
    break;
  }
  if (tail <= 0 || tail > max_tail || tail >= cols || tail == copy) return false;
  const int prefix = cols - tail;
  if (suffix[copy - tail - 1] != 0.0 || (prefix & 1)) return false;
  *pairs = prefix / 2;
  return *pairs >= min_pairs;
}

// The epigraph attempt: true when the plan was rewritten (or the model was
// found infeasible).
bool try_epigraph(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  const DevCsr& A = lp.A;
  int P = 0;
  if (!epigraph_layout(lp, p, &P)) return false;
  auto s = ctx().stream;
  const int rows = A.rows, cols = A.cols;
  // Probes (quick_probe_..._epigraph_impl, :859-924).
  {
    const int probes = std::max(1, std::min(P, p.piecewise_linear_reformulation_variable_pair_epigraph_probe_pairs));
    DBuf<int32_t> st(2, s);
    st.zero();
    GPP_LAUNCH(epi_pair_probe, grid_stride_blocks(probes), kThreads, 0, s, P, cols, probes, lp.AT.ptr, lp.AT.idx,
               lp.AT.val, A.ptr, A.idx, A.val, lp.AL, lp.AU, lp.c, lp.l, lp.u, st.p);
    if (!merge_rows_dense_enough(A, lp.AL, lp.AU, P, s, st.p, st.p + 1)) return false;
  }
  const int max_terms = std::max(1, std::min(kMaxQuotientTerms,
                                             p.piecewise_linear_reformulation_variable_pair_epigraph_max_quotient_terms_per_row));
  const EpiArgs g{A.ptr, A.idx, A.val, lp.AL, lp.AU, lp.c, lp.l, lp.u, rows, cols, P, max_terms};
  DBuf<double> shift(size_t(P), s), lower_sum(size_t(P), s), gcoef(size_t(P), s);
  DBuf<unsigned long long> edge(size_t(rows), s);
  DBuf<int32_t> g_by_row(size_t(rows), s), g_row(size_t(P), s), tail(size_t(P), s), st(4, s);
  st.zero();
  GPP_LAUNCH(fill_minus_one, grid_stride_blocks(P), kThreads, 0, s, g_row.p, P);
  GPP_LAUNCH(epi_columns, grid_stride_blocks(std::max(P, cols - 2 * P)), kThreads, 0, s, g, shift.p, lower_sum.p, st.p);
  GPP_LAUNCH(epi_classify, grid_stride_blocks(rows), kThreads, 0, s, g, shift.p, edge.p, g_by_row.p, g_row.p, tail.p,
             gcoef.p, st.p + 1, st.p);
  int32_t census[3];
  check(cudaMemcpyAsync(ctx().host_status, st.p, sizeof(int32_t) * 3, cudaMemcpyDeviceToHost, s), "epigraph census");
  ctx().sync("epigraph census");
  std::copy(ctx().host_status, ctx().host_status + 3, census);
  const int edges = census[1];
  if (census[0] != 0 || census[2] != P) return false;
  const double potential = double(std::min(edges, P - 1)) / double(P);
  if (edges < std::max(1, p.piecewise_linear_reformulation_variable_pair_epigraph_min_pairs) ||
      potential < p.piecewise_linear_reformulation_variable_pair_epigraph_min_potential_gain)
    return false;
  DBuf<int32_t> parent;
  const int comps = components(P, rows, edge.p, parent, s);
  if (comps <= 0) return false;
  const double actual = 1.0 - double(comps) / double(P);
  if (actual < p.piecewise_linear_reformulation_variable_pair_epigraph_min_actual_gain) return false;
  DBuf<uint64_t> keys(size_t(P), s);
  DBuf<int32_t> order(size_t(P), s), size(size_t(P), s);
  DBuf<double> plus_up(size_t(P), s), minus_up(size_t(P), s);
  GPP_LAUNCH(component_keys, grid_stride_blocks(P), kThreads, 0, s, P, parent.p, keys.p, order.p);
  radix_sort_pairs(keys.p, order.p, P, s);
  GPP_LAUNCH(epi_aggregate, grid_stride_blocks(P), kThreads, 0, s, P, keys.p, order.p, lp.u, size.p, plus_up.p,
             minus_up.p);
  DBuf<int32_t> vst(1, s);
  vst.zero();
  GPP_LAUNCH(epi_validate, grid_stride_blocks(P), kThreads, 0, s, g, parent.p, g_row.p, tail.p, gcoef.p, shift.p,
             lower_sum.p, plus_up.p, minus_up.p, vst.p);
  // Rewrite (build_..._epigraph_plan, :1155-1300) into scratch.
  DBuf<int32_t> counts(size_t(rows) + 1, s), removed(2, s);
  DBuf<uint8_t> keep(size_t(rows), s);
  DBuf<double> al(size_t(rows), s), au(size_t(rows), s);
  removed.zero();
  GPP_LAUNCH(epi_rows, grid_stride_blocks(rows), kThreads, 0, s, g, parent.p, size.p, shift.p, edge.p, g_by_row.p,
             p.feasibility_tol, RowOut{counts.p, keep.p, al.p, au.p}, removed.p, removed.p + 1);
  int32_t vfail = 0, rstatus = 0;
  std::tie(vfail, rstatus) = read_scalars(vst.p, removed.p + 1);
  if (vfail) return false;
  if (rstatus & 32) return false;
  if (rstatus & 1) {
    plan.has_infeasible = true;
    return true;
  }
  DevCsr out;
  out.rows = rows;
  out.cols = cols;
  out.ptr = dalloc<offset_t>(size_t(rows) + 1);
  exclusive_scan_i32(counts.p, out.ptr, rows, s);
  int32_t nnz = 0, nremoved = 0;
  std::tie(nnz, nremoved) = read_scalars(out.ptr + rows, removed.p);
  out.nnz = nnz;
  out.idx = dalloc<int32_t>(size_t(nnz));
  out.val = dalloc<double>(size_t(nnz));
  GPP_LAUNCH(epi_fill, grid_stride_blocks(rows), kThreads, 0, s, g, parent.p, size.p, shift.p, tail.p, edge.p,
             g_by_row.p, out.ptr, out.idx, out.val);
  GPP_LAUNCH(epi_columns_apply, grid_stride_blocks(P), kThreads, 0, s, P, parent.p, plus_up.p, minus_up.p,
             plan.keep_col.p, plan.c.p, plan.l.p, plan.u.p);
  GPP_LAUNCH(commit_rows, grid_stride_blocks(rows), kThreads, 0, s, rows, keep.p, al.p, au.p, plan.keep_row.p,
             plan.AL.p, plan.AU.p);
  plan.new_A = out;
  plan.has_new_A = true;
  plan.has_change = true;
  plan.has_row_action = nremoved > 0;
  plan.has_col_action = comps < P;
  plan.varpair = make_recovery(P, parent.p, lp.l, false, s);
  return true;
}

// ---- shifted antipodal ------------------------------------------------------------------------

bool try_shifted_antipodal(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  const DevCsr& A = lp.A;
  const int rows = A.rows, cols = A.cols;
  if (cols <= 0 || (cols & 1) || rows <= 0) return false;
  const int P = cols / 2;
  if (P < std::max(1, p.piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs)) return false;
  auto s = ctx().stream;
  {
    const int probes =
        std::max(1, std::min(P, p.piecewise_linear_reformulation_variable_pair_shifted_antipodal_probe_pairs));
    DBuf<int32_t> st(2, s);
    st.zero();
    GPP_LAUNCH(anti_pair_probe, grid_stride_blocks(probes), kThreads, 0, s, P, probes, lp.AT.ptr, lp.AT.idx,
               lp.AT.val, lp.c, lp.l, lp.u, st.p);
    if (!merge_rows_dense_enough(A, lp.AL, lp.AU, P, s, st.p, st.p + 1)) return false;
  }
  const int max_terms =
      std::max(1, std::min(kMaxQuotientTerms,
                           p.piecewise_linear_reformulation_variable_pair_shifted_antipodal_max_quotient_terms_per_row));
  DBuf<double> shift(size_t(P), s), constant(size_t(P), s);
  DBuf<unsigned long long> edge(size_t(rows), s);
  DBuf<int32_t> st(2, s);
  st.zero();
  GPP_LAUNCH(anti_columns, grid_stride_blocks(P), kThreads, 0, s, P, lp.c, lp.l, lp.u, shift.p, constant.p, st.p);
  GPP_LAUNCH(anti_classify, grid_stride_blocks(rows), kThreads, 0, s, A.ptr, A.idx, A.val, lp.AL, lp.AU, shift.p, rows,
             P, max_terms, edge.p, st.p + 1, st.p);
  int32_t status = 0, edges = 0;
  std::tie(status, edges) = read_scalars(st.p, st.p + 1);
  if (status != 0 || edges < 1) return false;
  const double potential = double(std::min(edges, P - 1)) / double(P);
  if (edges < std::max(1, p.piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs) ||
      potential < p.piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_potential_gain)
    return false;
  DBuf<int32_t> parent;
  const int comps = components(P, rows, edge.p, parent, s);
  DBuf<int32_t> vst(1, s);
  vst.zero();
  GPP_LAUNCH(anti_verify, grid_stride_blocks(rows), kThreads, 0, s, rows, edge.p, parent.p, shift.p, vst.p);
  if (read_scalar(vst.p) != 0 || comps <= 0) return false;
  const double actual = 1.0 - double(comps) / double(P);
  if (actual < p.piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_actual_gain) return false;
  DBuf<uint64_t> keys(size_t(P), s);
  DBuf<int32_t> order(size_t(P), s);
  DBuf<double> plus_cap(size_t(P), s), minus_cap(size_t(P), s), rho(size_t(P), s);
  GPP_LAUNCH(component_keys, grid_stride_blocks(P), kThreads, 0, s, P, parent.p, keys.p, order.p);
  radix_sort_pairs(keys.p, order.p, P, s);
  GPP_LAUNCH(anti_aggregate, grid_stride_blocks(P), kThreads, 0, s, P, keys.p, order.p, lp.c, lp.l, lp.u, plus_cap.p,
             minus_cap.p, rho.p, vst.p);
  if (read_scalar(vst.p) != 0) return false;
  // The objective constant sum_i rho_i (l_p + l_m), in pair order.
  const double delta = det_sum(constant.p, P, s);
  if (!std::isfinite(delta) || !std::isfinite(lp.obj + delta)) return false;
  DBuf<int32_t> counts(size_t(rows) + 1, s), removed(2, s);
  DBuf<uint8_t> keep(size_t(rows), s);
  DBuf<double> al(size_t(rows), s), au(size_t(rows), s);
  removed.zero();
  GPP_LAUNCH(anti_rows, grid_stride_blocks(rows), kThreads, 0, s, A.ptr, A.idx, A.val, lp.AL, lp.AU, rows, parent.p,
             shift.p, edge.p, p.feasibility_tol, RowOut{counts.p, keep.p, al.p, au.p}, removed.p, removed.p + 1);
  DevCsr out;
  out.rows = rows;
  out.cols = cols;
  out.ptr = dalloc<offset_t>(size_t(rows) + 1);
  exclusive_scan_i32(counts.p, out.ptr, rows, s);
  int32_t nnz = 0, rstatus = 0;
  std::tie(nnz, rstatus) = read_scalars(out.ptr + rows, removed.p + 1);
  if (rstatus != 0) {
    // The reference reports any failed row rewrite as infeasible (:1020-1027).
    free_csr(out);
    plan.has_infeasible = true;
    return true;
  }
  const int32_t nremoved = read_scalar(removed.p);
  out.nnz = nnz;
  out.idx = dalloc<int32_t>(size_t(nnz));
  out.val = dalloc<double>(size_t(nnz));
  GPP_LAUNCH(anti_fill, grid_stride_blocks(rows), kThreads, 0, s, A.ptr, A.idx, A.val, rows, P, parent.p, shift.p,
             out.ptr, out.idx, out.val);
  plan.varpair = make_recovery(P, parent.p, lp.l, true, s);
  GPP_LAUNCH(anti_columns_apply, grid_stride_blocks(P), kThreads, 0, s, P, parent.p, plus_cap.p, minus_cap.p, rho.p,
             plan.keep_col.p, plan.c.p, plan.l.p, plan.u.p);
  GPP_LAUNCH(commit_rows, grid_stride_blocks(rows), kThreads, 0, s, rows, keep.p, al.p, au.p, plan.keep_row.p,
             plan.AL.p, plan.AU.p);
  plan.new_A = out;
  plan.has_new_A = true;
  plan.obj_delta += delta;
  plan.has_change = true;
  plan.has_row_action = nremoved > 0;
  plan.has_col_action = comps < P;
  return true;
}

}  // namespace

void rule_variable_pair(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  if (!p.enable_piecewise_linear_reformulation_variable_pair || lp.m() <= 0 || lp.n() <= 0) return;
  if (try_epigraph(plan, lp, p)) return;
  try_shifted_antipodal(plan, lp, p);
}

}  // namespace gpp
