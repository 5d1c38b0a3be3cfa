// Postsolve: scatter the reduced solution to the original index space,
// restore fixed values, replay the tape in reverse (primal pass, then dual
// pass), and project reduced costs z = proj(c - A^T y) for the columns no
// record recovered exactly.
//
// Reference: postsolve_gpu (cpp/src/presolve/gpu_postsolve.cu:535-670) and the
// record handlers in cpp/src/presolve/postsolve/*.cuh.  The per-record
// arithmetic is the reference's; records are replayed in reverse
// chronological order by one thread per segment walk (the reference's serial
// interpreter), and the closing projection runs one thread per column.
#include "presolve.hpp"
#include "sort.hpp"

namespace gpp {

namespace {

constexpr double kTol = 1e-7;
// Tapes shorter than this replay on one thread (the grouping costs more).
constexpr int64_t kParallelMinRecords = 1024;
enum : int {
  kFixedVariable = 0, kInfiniteBoundDualFix = 1, kSingletonColumnSubstitution = 2, kParallelColumn = 3,
  kParallelRow = 4, kDeletedRow = 5, kRowDualShift = 10, kRowImpliedBoundChange = 12, kDoubletonEquation = 13,
  kFmeCol = 14
};

__device__ __forceinline__ bool pfin(double x) { return x > -INFINITY && x < INFINITY; }
__device__ __forceinline__ bool at_lower(double x, double l, double tol) { return pfin(l) && x <= l + tol; }
__device__ __forceinline__ bool at_upper(double x, double u, double tol) { return pfin(u) && x >= u - tol; }
__device__ __forceinline__ double clamp_inf(double x, double lo, double hi) {
  double y = x;
  if (pfin(lo)) y = fmax(y, lo);
  if (pfin(hi)) y = fmin(y, hi);
  return y;
}

struct Model {
  const offset_t *A_ptr, *AT_ptr;
  const int32_t *A_idx, *AT_idx;
  const double *A_val, *AT_val, *c, *l, *u;
  bool present;
};
struct Sol {
  double *x, *y, *z;
  uint8_t* got;
};

__device__ double merged_source_value(double lo, double hi, double tol) {
  if (isfinite(lo) && isfinite(hi)) return 0.5 * (lo + hi);
  if (isfinite(lo)) { if (0.0 > lo + tol) return 0.0; return lo + fmax(1.0, fabs(lo) * fmax(tol, 1.0e-12)); }
  if (isfinite(hi)) { if (0.0 < hi - tol) return 0.0; return hi - fmax(1.0, fabs(hi) * fmax(tol, 1.0e-12)); }
  return 0.0;
}

__device__ void replay_record(int type, const int32_t* id, int64_t ni, const double* v, int64_t nv, Sol s,
                              const Model& M, bool primal, bool dual) {
  const double tol = kTol;
  double* x = s.x;
  double* y = s.y;
  double* z = s.z;
  if (type == kParallelColumn) {
    // replay_parallel_column (postsolve_parallel_columns.cuh:101-131).
    const int from = id[0], to = id[1];
    const double r = v[0], lo = v[1], hi = v[2], tl = v[3], tu = v[4];
    if (primal) {
      const double yv = x[to], zt = z ? z[to] : 0.0;
      double slo = lo, shi = hi;
      if (isfinite(tu)) { const double b = (yv - tu) / r; if (r > 0.0) slo = fmax(slo, b); else shi = fmin(shi, b); }
      if (isfinite(tl)) { const double b = (yv - tl) / r; if (r > 0.0) shi = fmin(shi, b); else slo = fmax(slo, b); }
      double lower = -INFINITY, upper = INFINITY;
      if (r > 0.0) { if (isfinite(tl) && isfinite(lo)) lower = tl + r * lo; }
      else if (isfinite(tl) && isfinite(hi)) lower = tl + r * hi;
      if (r > 0.0) { if (isfinite(tu) && isfinite(hi)) upper = tu + r * hi; }
      else if (isfinite(tu) && isfinite(lo)) upper = tu + r * lo;
      double xf;
      if (zt > tol && isfinite(lower) && fabs(yv - lower) <= tol) xf = r > 0.0 ? lo : hi;
      else if (zt < -tol && isfinite(upper) && fabs(yv - upper) <= tol) xf = r > 0.0 ? hi : lo;
      else xf = merged_source_value(slo, shi, tol);
      x[from] = xf;
      x[to] = yv - r * xf;
    }
    if (dual && z) { z[from] = r * z[to]; s.got[from] = 1; }
  } else if (type == kDoubletonEquation) {
    // replay_doubleton_equation (postsolve_doubleton_equations.cuh:88-172).
    const int ec = id[0], kc = id[1], row = id[2];
    const double ecoef = v[0], kcoef = v[1], rhs = v[2], eobj = v[9];
    const double alpha = -kcoef / ecoef, beta = rhs / ecoef;
    if (primal) x[ec] = beta + alpha * x[kc];
    if (dual && z && y && M.present) {
      const double okl = v[5], oku = v[6], nkl = v[7], nku = v[8];
      const double lsrc = nv >= 11 ? v[10] : 0.0, usrc = nv >= 12 ? v[11] : 0.0;
      double zk = 0.0, ze = 0.0;
      const double xk = x[kc], zkh = z[kc];
      if (fabs(alpha) <= tol) { zk = zkh; ze = 0.0; }
      else {
        const bool al = pfin(nkl) && xk <= nkl + tol, au = pfin(nku) && xk >= nku - tol;
        if (!al && !au) { zk = 0.0; ze = 0.0; }
        else {
          double src = al ? lsrc : usrc;
          if (src == 0.0) {
            if (al) src = (pfin(okl) && fabs(nkl - okl) <= tol) ? 1.0 : 2.0;
            else src = (pfin(oku) && fabs(nku - oku) <= tol) ? 1.0 : 2.0;
          }
          if (src == 2.0) { zk = 0.0; ze = zkh / alpha; } else { zk = zkh; ze = 0.0; }
        }
      }
      double sum_other = 0.0;
      if (ni >= 4 && nv >= 12) {
        const int cnt = id[3];
        for (int q = 0; q < cnt; ++q) sum_other += v[12 + q] * y[id[4 + q]];
        y[row] = (eobj - sum_other - ze) / ecoef;
      } else {
        for (offset_t q = M.AT_ptr[ec]; q < M.AT_ptr[ec + 1]; ++q)
          if (M.AT_idx[q] != row) sum_other += M.AT_val[q] * y[M.AT_idx[q]];
        y[row] = (M.c[ec] - sum_other - ze) / ecoef;
      }
      z[kc] = zk; z[ec] = ze; s.got[kc] = 1; s.got[ec] = 1;
    } else if (dual) {
      if (z) { z[ec] = 0.0; s.got[ec] = 1; }
      if (y && row >= 0) y[row] = eobj / ecoef;
    }
  } else if (type == kSingletonColumnSubstitution) {
    // replay_singleton_column_substitution (postsolve_singleton_columns.cuh:8-50).
    const int ec = id[0], row = id[1], cnt = id[2];
    const double piv = v[0], rhs = v[1], eobj = v[4];
    const bool deleted = v[5] != 0.0;
    double part = 0.0;
    for (int q = 0; q < cnt; ++q) part += v[6 + q] * x[id[3 + q]];
    if (primal) x[ec] = (rhs - part) / piv;
    if (dual && y && row >= 0) { if (deleted) y[row] = eobj / piv; else y[row] += eobj / piv; }
    if (dual && z) { z[ec] = deleted || !y ? 0.0 : eobj - piv * y[row]; s.got[ec] = 1; }
  } else if (type == kFixedVariable) {
    // replay_fixed_variable (postsolve_fixed_variables.cuh:8-40).
    const int col = id[0];
    if (primal) x[col] = v[0];
    if (dual && z) {
      double zj = v[1];
      if (y) for (int64_t q = 1; q < ni; ++q) zj -= v[2 + (q - 1)] * y[id[q]];
      z[col] = zj;
      s.got[col] = 1;
    }
  } else if (type == kInfiniteBoundDualFix) {
    // replay_infinite_bound_dual_fix (postsolve_fixed_variables.cuh:42-89).
    const bool pos = id[0] > 0;
    const int col = id[1], nrows = id[2];
    double ext = v[0];
    int64_t ip = 3, vp = 1;
    if (primal) {
      for (int r = 0; r < nrows; ++r) {
        const int len = id[ip];
        double side = v[vp], coeff = 0.0;
        for (int q = 0; q < len; ++q) {
          const int c2 = id[ip + 1 + q];
          const double a = v[vp + 1 + q];
          if (c2 == col) coeff = a; else side -= a * x[c2];
        }
        const double cand = side / coeff;
        ext = pos ? fmax(ext, cand) : fmin(ext, cand);
        ip += len + 1;
        vp += len + 1;
      }
      x[col] = ext;
    }
    if (dual && z) { z[col] = 0.0; s.got[col] = 1; }
  } else if (type == kFmeCol) {
    // replay_projected_column (postsolve_projected_variables.cuh:10-66):
    // x = max of the lower expressions (else min of the upper ones, else 0);
    // the column's reduced cost and its rows' duals are zero.
    const int K = id[0], col = id[1], L = id[3 + K];
    int64_t meta = 4 + K, at = 4 + K + 2 * int64_t(L), vp = 0;
    if (primal) {
      double lo = -INFINITY, hi = INFINITY;
      bool has_lo = false, has_hi = false;
      for (int e = 0; e < L; ++e) {
        const int orient = id[meta++];
        const int len = id[meta++];
        double cand = v[vp];
        for (int t = 0; t < len; ++t) cand += v[vp + 1 + t] * x[id[at++]];
        if (orient > 0) { lo = fmax(lo, cand); has_lo = true; } else { hi = fmin(hi, cand); has_hi = true; }
        vp += 1 + len;
      }
      x[col] = has_lo ? lo : (has_hi ? hi : 0.0);
    }
    if (dual && z) { z[col] = 0.0; s.got[col] = 1; }
    if (dual && y) for (int t = 0; t < K; ++t) y[id[2 + t]] = 0.0;
  } else if (dual && type == kRowDualShift) {
    if (y) y[id[0]] += v[0];
  } else if (dual && type == kParallelRow && ni >= 2 && nv >= 5) {
    // replay_parallel_row (postsolve_parallel_rows.cuh:170-250).
    const int kept = id[0], del = id[1];
    const double r = v[0], kal = v[1], kau = v[2], dal = v[3], dau = v[4];
    if (fabs(r) <= tol || !y) return;
    double dsl = dal * r, dsu = dau * r;
    if (r < 0.0) { const double t = dsl; dsl = dsu; dsu = t; }
    if (dsl <= kal + tol && kau <= dsu + tol) { y[del] = 0.0; return; }
    if (!M.present) return;
    auto act = [&](int row) {
      double a = 0.0;
      for (offset_t q = M.A_ptr[row]; q < M.A_ptr[row + 1]; ++q) a += M.A_val[q] * x[M.A_idx[q]];
      return a;
    };
    auto state = [&](double a, double lo, double hi) {
      const bool L = pfin(lo) && a <= lo + tol, U = pfin(hi) && a >= hi - tol;
      return L && U ? 3 : L ? 1 : U ? 2 : 0;
    };
    const int ks = state(act(kept), kal, kau), ds = state(act(del), dal, dau);
    double ydl, ydh, ypl, yph;
    if (ds == 3) { ydl = -INFINITY; ydh = INFINITY; } else if (ds == 1) { ydl = 0.0; ydh = INFINITY; }
    else if (ds == 2) { ydl = -INFINITY; ydh = 0.0; } else { ydl = 0.0; ydh = 0.0; }
    const double pv = r * y[kept];
    if (ks == 3) { ypl = -INFINITY; yph = INFINITY; }
    else if (ks == 0) { ypl = pv; yph = pv; }
    else if (ks == 1) { if (r > 0.0) { ypl = -INFINITY; yph = pv; } else { ypl = pv; yph = INFINITY; } }
    else { if (r > 0.0) { ypl = pv; yph = INFINITY; } else { ypl = -INFINITY; yph = pv; } }
    const double sl = fmax(ydl, ypl), sh = fmin(ydh, yph);
    if (sl <= sh + tol) {
      const double yd = clamp_inf(0.0, sl, sh);
      y[kept] = y[kept] - yd / r;
      y[del] = yd;
      return;
    }
    const double yb = y[kept];
    double yp = yb, yd = 0.0;
    bool ok;
    if (fabs(yb) <= tol) { yp = 0.0; yd = 0.0; ok = true; }
    else {
      const double bl = fmax(kal, dsl), bu = fmin(kau, dsu);
      if (!(bl <= bu + tol)) ok = false;
      else {
        const bool lt = bl > kal + tol, ut = bu < kau - tol;
        if (lt && ut) ok = false;
        else if (!lt && !ut) { yp = yb; yd = 0.0; ok = true; }
        else {
          ok = true;
          if (yb > 0.0) { if (lt) { yp = 0.0; yd = r * yb; } else { yp = yb; yd = 0.0; } }
          else { if (lt) { yp = yb; yd = 0.0; } else { yp = 0.0; yd = r * yb; } }
        }
      }
    }
    if (ok) { y[kept] = yp; y[del] = yd; }
  } else if (dual && type == kDeletedRow && M.present && ni >= 2 && nv >= 3) {
    // replay_deleted_singleton_row (postsolve_singleton_rows.cuh:8-96).
    const int row = id[0], col = id[1];
    const double oal = v[0], oau = v[1], a = v[2];
    if (fabs(a) <= tol) return;
    double g = M.c[col];
    for (offset_t q = M.AT_ptr[col]; q < M.AT_ptr[col + 1]; ++q)
      if (M.AT_idx[q] != row && y) g -= M.AT_val[q] * y[M.AT_idx[q]];
    const double xj = x[col], zb = z[col], ra = a * xj;
    const bool rl = isfinite(oal) && ra <= oal + tol, ru = isfinite(oau) && ra >= oau - tol;
    double lo = -INFINITY, hi = INFINITY;
    if (!(rl && ru)) {
      if (rl) { if (a > 0.0) hi = g; else lo = g; }
      else if (ru) { if (a > 0.0) lo = g; else hi = g; }
      else { lo = g; hi = g; }
    }
    const bool L = at_lower(xj, M.l[col], tol), U = at_upper(xj, M.u[col], tol);
    double zl = lo, zh = hi;
    if (!L && !U) {
      if ((isfinite(lo) && lo > tol) || (isfinite(hi) && hi < -tol)) { zl = g; zh = g; } else { zl = 0.0; zh = 0.0; }
    } else if (L && !U) zl = fmax(zl, 0.0);
    else if (!L && U) zh = fmin(zh, 0.0);
    if (isfinite(zl) && isfinite(zh) && zl > zh + tol) return;
    const double zn = clamp_inf(zb, zl, zh);
    z[col] = zn;
    if (y) y[row] = (g - zn) / a;
    s.got[col] = 1;
  } else if (dual && type == kRowImpliedBoundChange && M.present && ni >= 2) {
    // replay_row_implied_bound_change (postsolve_bound_strengthening.cuh:8-76).
    const int col = id[0], row = id[1];
    if (!s.got[col]) return;
    const double ol = v[0], ou = v[1], nl = v[2], nu = v[3];
    const bool lc = nl > ol + tol, uc = nu < ou - tol;
    if (lc == uc) return;
    const double ib = lc ? nl : nu, other = lc ? ou : ol;
    const bool other_lower = !lc;
    const double xj = x[col], zj = z[col];
    if (pfin(other) && fabs(xj - other) <= tol) {
      const bool ok = other_lower ? (zj >= -tol) : (zj <= tol);
      if (ok) return;
    }
    if (fabs(xj - ib) > tol) return;
    double aij = 0.0;
    for (offset_t q = M.A_ptr[row]; q < M.A_ptr[row + 1]; ++q)
      if (M.A_idx[q] == col) { aij = M.A_val[q]; break; }
    if (fabs(aij) <= tol) return;
    if (y) y[row] += zj / aij;
    for (offset_t q = M.A_ptr[row]; q < M.A_ptr[row + 1]; ++q) {
      const int kc = M.A_idx[q];
      if (kc == col || !s.got[kc]) continue;
      z[kc] -= (M.A_val[q] / aij) * zj;
    }
    z[col] = 0.0;
    s.got[col] = 1;
  }
}

struct SegView {
  const int32_t* types;
  const int64_t* is;
  const int64_t* vs;
  const int32_t* idx;
  const double* val;
  int64_t count;
};

// The reference's serial interpreter: one thread walks records [lo, hi) of a
// segment backwards.
__global__ void replay_serial(SegView t, Sol s, Model M, int primal, int dual, int64_t lo, int64_t hi) {
  if (blockIdx.x || threadIdx.x) return;
  for (int64_t k = hi - 1; k >= lo; --k)
    replay_record(t.types[k], t.idx + t.is[k], t.is[k + 1] - t.is[k], t.val + t.vs[k], t.vs[k + 1] - t.vs[k], s, M,
                  primal != 0, dual != 0);
}

__global__ void scatter(double* __restrict__ dst, const double* __restrict__ src, const int32_t* __restrict__ map,
                        int32_t n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[map[i]] = src[i];
}
__global__ void mark(uint8_t* __restrict__ got, const int32_t* __restrict__ map, int32_t n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) got[map[i]] = 1;
}
__global__ void restore_fixed(double* __restrict__ x, const int32_t* __restrict__ idx, const double* __restrict__ val,
                              int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[idx[i]] = val[i];
}
__global__ void mark_protected(SegView t, uint8_t* __restrict__ prot, int n) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < t.count; k += int64_t(gridDim.x) * blockDim.x) {
    const int type = t.types[k];
    const int32_t* id = t.idx + t.is[k];
    int a = -1, b = -1;
    if (type == kSingletonColumnSubstitution || type == kParallelColumn) a = id[0];
    if (type == kDoubletonEquation) { a = id[0]; b = id[1]; }
    if (type == kInfiniteBoundDualFix) a = id[1];
    if (a >= 0 && a < n) prot[a] = 1;
    if (b >= 0 && b < n) prot[b] = 1;
  }
}
// project_column_duals_from_original (gpu_postsolve.cu:355-398, postsolve_common.cuh:59-94):
// warp per column, A^T y summed sequentially by lane 0 in stored order.
__global__ void project_duals(int n, const uint8_t* __restrict__ prot, Model M, const double* __restrict__ x,
                              const double* __restrict__ y, double* __restrict__ z) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (prot[j]) continue;
    double aty = 0.0;
    for (offset_t q = M.AT_ptr[j]; q < M.AT_ptr[j + 1]; ++q) aty += M.AT_val[q] * y[M.AT_idx[q]];
    const double r = M.c[j] - aty;
    const bool L = at_lower(x[j], M.l[j], kTol), U = at_upper(x[j], M.u[j], kTol);
    double zj;
    if (L && U) zj = r; else if (!L && !U) zj = 0.0; else if (L) zj = fmax(r, 0.0); else zj = fmin(r, 0.0);
    const double eps = fmin(kTol, 1.0e-12);
    if (zj > eps && !isfinite(M.l[j])) zj = 0.0;
    else if (zj < -eps && !isfinite(M.u[j])) zj = 0.0;
    z[j] = zj;
  }
}

SegView view(const PostsolveSegment& s) { return {s.types.p, s.is.p, s.vs.p, s.idx.p, s.val.p, s.count}; }

// ---- component-parallel replay ----------------------------------------------
//
// Replaying the tape in reverse chronological order is equivalent to
// replaying, in that order, each group of records that share a resource one
// of them writes, with the groups independent of one another.  Resources are
// the columns (x, z and the retrieval flag together) and the rows (y) of the
// original model; per pass only what that pass reads or writes counts (x is
// read-only in the dual pass, y and z untouched in the primal pass).  Records
// that do nothing in a pass (variable bound changes, and the dual-only records
// in the primal pass) drop out.  Groups come from a lock-free union-find over
// the records; each group is replayed by one thread, newest record first.

struct TapeView {
  const SegView* segs;       // device array
  const int64_t* starts;     // global index of each segment's first record, count+1 entries
  int nseg;
  int64_t total;
  __device__ void at(int64_t g, int& type, const int32_t*& id, int64_t& ni, const double*& v, int64_t& nv) const {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (starts[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const SegView& t = segs[lo];
    const int64_t k = g - starts[lo];
    type = t.types[k];
    id = t.idx + t.is[k];
    ni = t.is[k + 1] - t.is[k];
    v = t.val + t.vs[k];
    nv = t.vs[k + 1] - t.vs[k];
  }
};

__device__ __forceinline__ bool replays_in(int type, bool dual) {
  if (type == kFixedVariable || type == kInfiniteBoundDualFix || type == kSingletonColumnSubstitution ||
      type == kParallelColumn || type == kDoubletonEquation || type == kFmeCol)
    return true;
  return dual && (type == kRowDualShift || type == kParallelRow || type == kDeletedRow || type == kRowImpliedBoundChange);
}

// Calls visit(resource, writes) for every resource the record touches in the
// pass; columns are 0..n-1, rows n..n+m-1.
template <class F>
__device__ void record_resources(int type, const int32_t* id, int64_t ni, int64_t nv, bool dual, int m, int n,
                                 const Model& M, F visit) {
  auto col = [&](int j, bool w) { if (j >= 0 && j < n) visit(j, w); };
  auto row = [&](int i, bool w) { if (i >= 0 && i < m) visit(n + i, w); };
  if (!dual) {
    switch (type) {
      case kFixedVariable: col(id[0], true); break;
      case kInfiniteBoundDualFix: {
        col(id[1], true);
        int64_t ip = 3;
        for (int r = 0; r < id[2] && ip < ni; ++r) {
          const int len = id[ip];
          for (int q = 0; q < len && ip + 1 + q < ni; ++q) col(id[ip + 1 + q], false);
          ip += len + 1;
        }
        break;
      }
      case kSingletonColumnSubstitution:
        col(id[0], true);
        for (int q = 0; q < id[2] && 3 + q < ni; ++q) col(id[3 + q], false);
        break;
      case kParallelColumn: col(id[0], true); col(id[1], true); break;
      case kDoubletonEquation: col(id[0], true); col(id[1], false); break;
      case kFmeCol:
        if (ni >= 4) {
          const int K = id[0];
          col(id[1], true);
          if (3 + K < ni) {
            const int terms = id[2 + K];
            const int64_t first = int64_t(4 + K) + 2 * int64_t(id[3 + K]);
            for (int t = 0; t < terms && first + t < ni; ++t) col(id[first + t], false);
          }
        }
        break;
      default: break;
    }
    return;
  }
  switch (type) {
    case kFixedVariable:
      col(id[0], true);
      for (int64_t q = 1; q < ni; ++q) row(id[q], false);
      break;
    case kInfiniteBoundDualFix: col(id[1], true); break;
    case kSingletonColumnSubstitution: col(id[0], true); row(id[1], true); break;
    case kParallelColumn: col(id[0], true); col(id[1], false); break;
    case kDoubletonEquation:
      col(id[0], true); col(id[1], true); row(id[2], true);
      if (ni >= 4 && nv >= 12) {
        for (int q = 0; q < id[3] && 4 + q < ni; ++q) row(id[4 + q], false);
      } else if (M.present && id[0] >= 0 && id[0] < n) {
        for (offset_t q = M.AT_ptr[id[0]]; q < M.AT_ptr[id[0] + 1]; ++q) row(M.AT_idx[q], false);
      }
      break;
    case kFmeCol:
      if (ni >= 2) {
        col(id[1], true);
        for (int t = 0; t < id[0] && 2 + t < ni; ++t) row(id[2 + t], true);
      }
      break;
    case kRowDualShift: row(id[0], true); break;
    case kParallelRow: if (ni >= 2) { row(id[0], true); row(id[1], true); } break;
    case kDeletedRow:
      if (ni >= 2) {
        row(id[0], true); col(id[1], true);
        if (M.present && id[1] >= 0 && id[1] < n)
          for (offset_t q = M.AT_ptr[id[1]]; q < M.AT_ptr[id[1] + 1]; ++q) row(M.AT_idx[q], false);
      }
      break;
    case kRowImpliedBoundChange:
      if (ni >= 2) {
        col(id[0], true); row(id[1], true);
        if (M.present && id[1] >= 0 && id[1] < m)
          for (offset_t q = M.A_ptr[id[1]]; q < M.A_ptr[id[1] + 1]; ++q) col(M.A_idx[q], true);
      }
      break;
    default: break;
  }
}

__global__ void cp_active(TapeView t, int dual, int64_t lo, int64_t hi, int32_t* __restrict__ flag) {
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < t.total; g += int64_t(gridDim.x) * blockDim.x) {
    int type;
    const int32_t* id;
    int64_t ni, nv;
    const double* v;
    t.at(g, type, id, ni, v, nv);
    flag[g] = g >= lo && g < hi && replays_in(type, dual != 0) ? 1 : 0;
  }
}

__global__ void cp_list(int64_t total, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                        int64_t* __restrict__ act, int32_t* __restrict__ parent) {
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x)
    if (flag[g]) { act[pos[g]] = g; parent[pos[g]] = pos[g]; }
}

// First writer of each resource owns it.
__global__ void cp_claim(TapeView t, const int64_t* __restrict__ act, int count, int dual, int m, int n, Model M,
                         int32_t* __restrict__ owner) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    int type;
    const int32_t* id;
    int64_t ni, nv;
    const double* v;
    t.at(act[q], type, id, ni, v, nv);
    record_resources(type, id, ni, nv, dual != 0, m, n, M, [&](int res, bool w) {
      if (w) atomicCAS(owner + res, -1, q);
    });
  }
}

__device__ __forceinline__ int uf_root(int32_t* parent, int a) {
  for (;;) {
    const int b = *(volatile int32_t*)(parent + a);
    if (b == a) return a;
    a = b;
  }
}
// Link the larger root under the smaller; a failed CAS means the root moved,
// so retry from the new roots.  Links always point to smaller indices, so no
// cycle can form and every retry makes progress.
__device__ void uf_unite(int32_t* parent, int a, int b) {
  for (;;) {
    a = uf_root(parent, a);
    b = uf_root(parent, b);
    if (a == b) return;
    const int hi = a > b ? a : b, lo = a > b ? b : a;
    if (atomicCAS(parent + hi, hi, lo) == hi) return;
  }
}

// Every record joins the owner of each resource it touches.
__global__ void cp_connect(TapeView t, const int64_t* __restrict__ act, int count, int dual, int m, int n, Model M,
                           const int32_t* __restrict__ owner, int32_t* __restrict__ parent) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    int type;
    const int32_t* id;
    int64_t ni, nv;
    const double* v;
    t.at(act[q], type, id, ni, v, nv);
    record_resources(type, id, ni, nv, dual != 0, m, n, M, [&](int res, bool) {
      const int o = owner[res];
      if (o >= 0 && o != q) uf_unite(parent, q, o);
    });
  }
}

__global__ void cp_keys(int count, const int32_t* __restrict__ parent, uint64_t* __restrict__ keys,
                        int32_t* __restrict__ vals) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    int r = q;
    while (parent[r] != r) r = parent[r];
    keys[q] = (uint64_t(uint32_t(r)) << 32) | uint32_t(q);
    vals[q] = q;
  }
}

__global__ void cp_heads(int count, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x)
    head[q] = q == 0 || (keys[q] >> 32) != (keys[q - 1] >> 32) ? 1 : 0;
}
__global__ void cp_starts(int count, const int32_t* __restrict__ head, const int32_t* __restrict__ hpos,
                          int32_t* __restrict__ start) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x)
    if (head[q]) start[hpos[q]] = q;
}

// One thread per group: its records (sorted ascending) replayed newest first.
__global__ void cp_replay(TapeView t, const int64_t* __restrict__ act, const uint64_t* __restrict__ keys,
                          const int32_t* __restrict__ start, int groups, int count, Sol s, Model M, int primal,
                          int dual) {
  for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < groups; gi += gridDim.x * blockDim.x) {
    const int b = start[gi], e = gi + 1 < groups ? start[gi + 1] : count;
    for (int q = e - 1; q >= b; --q) {
      int type;
      const int32_t* id;
      int64_t ni, nv;
      const double* v;
      t.at(act[uint32_t(keys[q] & 0xffffffffu)], type, id, ni, v, nv);
      replay_record(type, id, ni, v, nv, s, M, primal != 0, dual != 0);
    }
  }
}

// Replays the records [lo, hi) of the whole tape (global indices).
void replay_parallel(const std::vector<PostsolveSegment>& segments, int m0, int n0, const Sol& s, const Model& M,
                     bool dual, cudaStream_t st, int64_t lo, int64_t hi) {
  std::vector<SegView> hv;
  std::vector<int64_t> hs{0};
  for (const auto& seg : segments) {
    if (!seg.count) continue;
    hv.push_back(view(seg));
    hs.push_back(hs.back() + seg.count);
  }
  const int64_t total = hs.back();
  if (!total) return;
  DBuf<SegView> segs(hv.size(), st);
  DBuf<int64_t> starts(hs.size(), st);
  check(cudaMemcpyAsync(segs.p, hv.data(), sizeof(SegView) * hv.size(), cudaMemcpyHostToDevice, st), "tape views");
  check(cudaMemcpyAsync(starts.p, hs.data(), sizeof(int64_t) * hs.size(), cudaMemcpyHostToDevice, st), "tape starts");
  const TapeView t{segs.p, starts.p, int(hv.size()), total};
  DBuf<int32_t> flag(size_t(total) + 1, st), pos(size_t(total) + 1, st);
  GPP_LAUNCH(cp_active, grid_stride_blocks(total), kThreads, 0, st, t, int(dual), lo, hi, flag.p);
  exclusive_scan_i32(flag.p, pos.p, total, st);
  const int count = read_scalar(pos.p + total);
  if (!count) return;
  DBuf<int64_t> act(size_t(count), st);
  DBuf<int32_t> parent(size_t(count), st), owner(size_t(m0) + size_t(n0), st);
  GPP_LAUNCH(cp_list, grid_stride_blocks(total), kThreads, 0, st, total, flag.p, pos.p, act.p, parent.p);
  check(cudaMemsetAsync(owner.p, 0xff, sizeof(int32_t) * (size_t(m0) + size_t(n0)), st), "owners");
  const int g = grid_stride_blocks(count);
  GPP_LAUNCH(cp_claim, g, kThreads, 0, st, t, act.p, count, int(dual), m0, n0, M, owner.p);
  GPP_LAUNCH(cp_connect, g, kThreads, 0, st, t, act.p, count, int(dual), m0, n0, M, owner.p, parent.p);
  DBuf<uint64_t> keys(size_t(count), st);
  DBuf<int32_t> vals(size_t(count), st), head(size_t(count) + 1, st), hpos(size_t(count) + 1, st);
  GPP_LAUNCH(cp_keys, g, kThreads, 0, st, count, parent.p, keys.p, vals.p);
  radix_sort_pairs(keys.p, vals.p, count, st);
  GPP_LAUNCH(cp_heads, g, kThreads, 0, st, count, keys.p, head.p);
  exclusive_scan_i32(head.p, hpos.p, count, st);
  const int groups = read_scalar(hpos.p + count);
  DBuf<int32_t> gstart(size_t(groups), st);
  GPP_LAUNCH(cp_starts, g, kThreads, 0, st, count, head.p, hpos.p, gstart.p);
  GPP_LAUNCH(cp_replay, grid_stride_blocks(groups, 128), 128, 0, st, t, act.p, keys.p, gstart.p, groups, count, s, M,
             int(!dual), int(dual));
}

// ---- piecewise-linear primal recoveries ---------------------------------------
// postsolve_piecewise_linear_reformulation_absolute_value.cu:9-105.

__global__ void restore_splits(double* __restrict__ x, const int32_t* __restrict__ t, const int32_t* __restrict__ e,
                               const double* __restrict__ rho, int k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
    const double tv = x[t[i]], ev = x[e[i]];
    x[t[i]] = tv + ev;
    x[e[i]] = (tv - ev) / rho[i];
  }
}
__global__ void restore_pairs(double* __restrict__ x, const int32_t* __restrict__ bound,
                              const int32_t* __restrict__ free_col, int k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) x[free_col[i]] = x[bound[i]];
}
__global__ void restore_links(double* __restrict__ x, const int32_t* __restrict__ slack, const int32_t* __restrict__ t,
                              const double* __restrict__ f, int k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) x[slack[i]] = f[i] * x[t[i]];
}
// One warp per group: slack = max(l_slack (0 when absent or not finite),
// max_k factor_k t_k).  fmax ignores NaN and is exact, so any order of the
// maximum gives the reference's value.
__global__ void restore_max_slacks(double* __restrict__ x, const int32_t* __restrict__ slack,
                                   const int32_t* __restrict__ start, const int32_t* __restrict__ t,
                                   const double* __restrict__ f, int groups, const double* __restrict__ lower) {
  const int lane = threadIdx.x & 31;
  for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < groups; g += (gridDim.x * blockDim.x) >> 5) {
    const int32_t sc = slack[g];
    double lb = lower ? lower[sc] : 0.0;
    if (!isfinite(lb)) lb = 0.0;
    double v = lb;
    for (int q = start[g] + lane; q < start[g + 1]; q += 32) v = fmax(v, f[q] * x[t[q]]);
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) x[sc] = v;
  }
}

// Roots' values first, then every member (restore_piecewise_linear_reformulation_variable_pair,
// postsolve_piecewise_linear_reformulation_variable_pair.cu:9-95).
__global__ void cache_pair_roots(double* __restrict__ pc, double* __restrict__ mc, const double* __restrict__ x,
                                 const int32_t* __restrict__ rp, const int32_t* __restrict__ rm, int k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
    pc[i] = x[rp[i]];
    mc[i] = x[rm[i]];
  }
}
__global__ void restore_pair_members(double* __restrict__ x, const int32_t* __restrict__ plus,
                                     const int32_t* __restrict__ minus, const double* __restrict__ ps,
                                     const double* __restrict__ ms, const double* __restrict__ pc,
                                     const double* __restrict__ mc, int k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
    x[plus[i]] = ps[i] + pc[i];
    x[minus[i]] = ms[i] + mc[i];
  }
}

}  // namespace

void restore_variable_pair(double* x, const VarPairRecovery& r, cudaStream_t st) {
  if (!r.count) return;
  DBuf<double> pc(size_t(r.count), st), mc(size_t(r.count), st);
  GPP_LAUNCH(cache_pair_roots, grid_stride_blocks(r.count), kThreads, 0, st, pc.p, mc.p, x, r.root_plus.p,
             r.root_minus.p, r.count);
  GPP_LAUNCH(restore_pair_members, grid_stride_blocks(r.count), kThreads, 0, st, x, r.plus.p, r.minus.p,
             r.plus_shift.p, r.minus_shift.p, pc.p, mc.p, r.count);
}

void restore_absolute_value(double* x, const AbsValueRecovery& r, const double* lower, cudaStream_t st) {
  GPP_LAUNCH(restore_splits, grid_stride_blocks(r.splits), kThreads, 0, st, x, r.split_t.p, r.split_e.p,
             r.split_rho.p, r.splits);
  GPP_LAUNCH(restore_pairs, grid_stride_blocks(r.pairs), kThreads, 0, st, x, r.pair_bound.p, r.pair_free.p, r.pairs);
  GPP_LAUNCH(restore_links, grid_stride_blocks(r.links), kThreads, 0, st, x, r.link_slack.p, r.link_t.p,
             r.link_factor.p, r.links);
  GPP_LAUNCH(restore_max_slacks, grid_stride_blocks(int64_t(r.max_groups) * 32), kThreads, 0, st, x, r.max_slack.p,
             r.max_start.p, r.max_t.p, r.max_factor.p, r.max_groups, lower);
}

void run_postsolve(const PresolveOutput& out, const double* x_red, const double* y_red, const double* z_red,
                   const gpp_lp* original, double* x, double* y, double* z, const double* lower) {
  const NvtxRange range("postsolve");
  if (!lower && original) lower = original->l;
  auto st = ctx().stream;
  const Record& r = out.record;
  const int m0 = r.m0, n0 = r.n0;
  if (n0) check(cudaMemsetAsync(x, 0, sizeof(double) * n0, st), "clear x");
  if (m0 && y) check(cudaMemsetAsync(y, 0, sizeof(double) * m0, st), "clear y");
  if (n0 && z) check(cudaMemsetAsync(z, 0, sizeof(double) * n0, st), "clear z");
  DBuf<uint8_t> got(size_t(std::max(n0, 1)), st);
  got.zero();
  if (x_red && r.n) GPP_LAUNCH(scatter, grid_stride_blocks(r.n), kThreads, 0, st, x, x_red, r.cols.p, r.n);
  if (y && y_red && r.m) GPP_LAUNCH(scatter, grid_stride_blocks(r.m), kThreads, 0, st, y, y_red, r.rows.p, r.m);
  if (z && z_red && r.n) GPP_LAUNCH(scatter, grid_stride_blocks(r.n), kThreads, 0, st, z, z_red, r.cols.p, r.n);
  if (r.n) GPP_LAUNCH(mark, grid_stride_blocks(r.n), kThreads, 0, st, got.p, r.cols.p, r.n);
  for (const auto& f : r.fixed)
    GPP_LAUNCH(restore_fixed, grid_stride_blocks(f.count), kThreads, 0, st, x, f.idx.p, f.val.p, f.count);
  Model M{};
  if (original) {
    M = Model{original->A.rowPtr, original->AT.rowPtr, original->A.colVal, original->AT.colVal, original->A.nzVal,
              original->AT.nzVal, original->c, original->l, original->u, true};
  }
  const Sol s{x, y, z, got.p};
  // Records [lo, hi) of the tape (global indices), newest first.
  auto replay = [&](int64_t lo, int64_t hi, bool dual) {
    if (lo >= hi) return;
    if (r.records < kParallelMinRecords) {
      int64_t end = r.records;
      for (auto it = r.segments.rbegin(); it != r.segments.rend(); ++it) {
        const int64_t begin = end - it->count;
        const int64_t a = std::max(lo, begin), b = std::min(hi, end);
        if (a < b) GPP_LAUNCH(replay_serial, 1, 1, 0, st, view(*it), s, M, !dual, dual, a - begin, b - begin);
        end = begin;
      }
    } else {
      replay_parallel(r.segments, m0, n0, s, M, dual, st, lo, hi);
    }
  };
  // Primal pass split at the piecewise-linear checkpoints, newest first: the
  // records after a checkpoint, then its recovery (postsolve_gpu,
  // gpu_postsolve.cu:637-663); the dual pass over the whole tape.
  int64_t range_end = r.records;
  for (auto it = r.timeline.rbegin(); it != r.timeline.rend(); ++it) {
    replay(it->tape_position, range_end, false);
    if (it->kind == 0) restore_absolute_value(x, r.absval[size_t(it->payload)], lower, st);
    else restore_variable_pair(x, r.varpair[size_t(it->payload)], st);
    range_end = it->tape_position;
  }
  replay(0, range_end, false);
  replay(0, r.records, true);
  if (original && y && z && n0) {
    DBuf<uint8_t> prot(size_t(n0), st);
    prot.zero();
    for (const auto& seg : r.segments)
      GPP_LAUNCH(mark_protected, grid_stride_blocks(seg.count), kThreads, 0, st, view(seg), prot.p, n0);
    GPP_LAUNCH(project_duals, grid_stride_blocks(n0), kThreads, 0, st, n0, prot.p, M, x, y, z);
  }
  ctx().sync("postsolve");
}

}  // namespace gpp
