// Doubleton-equation rule: substitute out one column of a two-entry equality.
//
// Reference: apply_rule_doubleton_equations -> _batch -> _batch_once
// (cpp/src/presolve/rules/rule_doubleton_equations.cu:1512-1812,1948-1957)
// with its kernels :150-271, :824-1489.  One call processes one batch:
//   * candidates: kept equality rows with exactly two live entries; the
//     eliminated column is chosen by column degree, then integral ratio, then
//     degree again (:170-214); pivot ratio within [1e-3, 1e3] (:161-168);
//     fill-in proxy over the sorted AT (:843-890, :960-987);
//   * 8 matching rounds in which a row that owns both of its unblocked
//     columns (smallest claiming row) is selected (:989-1027, :1604-1613);
//   * the batch runs only with >= min_selected_per_batch rows selected and a
//     selected/acceptable ratio >= min_selected_ratio (:1641-1655);
//   * substitution x_e = beta + alpha x_k with alpha = -a_k/a_e, beta =
//     rhs/a_e; mapped keep bounds; a keep column whose bounds close is fixed
//     at their midpoint instead (:1029-1117);
//   * the matrix is rebuilt with alpha * a_(r,e) merged into (r, k) and
//     entries |a| <= zero_tol dropped (:1191-1489); row sides shift by
//     a * beta (and a * value for fixed keep columns).
// With doubleton_equations_scan = 0 the reference's single-row mode runs
// instead: the smallest acceptable row alone, its column-stored matrix update
// and unfiltered row shifts (:273-512, :1814-2126).
// Where the reference sums with atomicAdd (row shifts, objective deltas),
// this engine sums in one fixed order: row shifts in stored column order per
// row, objective deltas in ascending row order of the batch.
#include <algorithm>
#include <climits>

#include "engine.cuh"
#include "sort.hpp"

namespace gpp {

namespace {

constexpr int kRounds = 8;
// Rows longer than this with at most kBlockMergeDeltas deltas are rebuilt by
// a block (dt_rebuild_block) instead of one lane.
constexpr int kBlockMergeRow = 64;
constexpr int kBlockMergeDeltas = 2048;
constexpr double kMaxPivotRatio = 1.0e3;
enum { kStInfeasible = 0, kStAny = 1, kStSubst = 2, kStFixed = 3, kStTouched = 4, kStWords = 5 };
enum : uint8_t { kPairNone = 0, kPairSubst = 1, kPairFixed = 2 };

// _kernel_doubleton_equations_live_col_nnz (:245-271).
__global__ void dt_col_nnz(int n, const offset_t* __restrict__ tptr, const int32_t* __restrict__ tidx,
                           const double* __restrict__ tval, const uint8_t* __restrict__ keep_row,
                           const uint8_t* __restrict__ keep_col, double zt, int32_t* __restrict__ col_nnz) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    int cnt = 0;
    if (keep_col[j])
      for (offset_t q = tptr[j]; q < tptr[j + 1]; ++q) cnt += keep_row[tidx[q]] && fabs(tval[q]) > zt ? 1 : 0;
    col_nnz[j] = cnt;
  }
}

__device__ bool integral_ratio(double num, double den, double tol) {
  // _is_integral_ratio_doubleton_equations (:150-159).
  if (fabs(den) <= tol) return false;
  const double r = fabs(num / den);
  if (!isfinite(r)) return false;
  return fabs(r - nearbyint(r)) <= tol;
}

__device__ __forceinline__ int next_live(const offset_t* tptr, const int32_t* tidx, const double* tval,
                                         const uint8_t* keep_row, double zt, int col, offset_t& pos) {
  while (pos < tptr[col + 1]) {
    const int r = tidx[pos];
    if (keep_row[r] && fabs(tval[pos]) > zt) return r;
    ++pos;
  }
  return INT_MAX;
}

// _doubleton_equations_fill_in_proxy_device_live (:843-890).
__device__ int fill_in_proxy(const offset_t* tptr, const int32_t* tidx, const double* tval, const uint8_t* keep_row,
                             double zt, int keep, int elim) {
  int fill = -1;
  offset_t jj = tptr[keep], kk = tptr[elim];
  const offset_t js = tptr[keep + 1], ks = tptr[elim + 1];
  if (js <= jj || ks <= kk) return fill;
  while (jj < js && kk < ks) {
    offset_t jl = jj, kl = kk;
    const int rj = next_live(tptr, tidx, tval, keep_row, zt, keep, jl);
    const int rk = next_live(tptr, tidx, tval, keep_row, zt, elim, kl);
    if (rj == INT_MAX || rk == INT_MAX) break;
    if (rj == rk) { jj = jl + 1; kk = kl + 1; }
    else if (rk < rj) { kk = kl + 1; ++fill; }
    else jj = jl + 1;
  }
  while (kk < ks) {
    offset_t kl = kk;
    if (next_live(tptr, tidx, tval, keep_row, zt, elim, kl) == INT_MAX) break;
    ++fill;
    kk = kl + 1;
  }
  return fill;
}

// _doubleton_equations_fill_in_proxy_device (:216-243): stored entries of AT,
// masks ignored (the single-row mode's proxy).
__device__ int fill_in_proxy_stored(const offset_t* tptr, const int32_t* tidx, int keep, int elim) {
  int fill = -1;
  offset_t jj = tptr[keep], kk = tptr[elim];
  const offset_t js = tptr[keep + 1], ks = tptr[elim + 1];
  if (js <= jj || ks <= kk) return fill;
  while (jj < js && kk < ks) {
    const int kr = tidx[jj], er = tidx[kk];
    if (kr == er) { ++jj; ++kk; }
    else if (er < kr) { ++kk; ++fill; }
    else ++jj;
  }
  return fill + int(ks - kk);
}

// Candidates and acceptance (:892-987; single-row mode :273-363), one thread
// per row.  Live selects the batch mode's masked fill-in proxy.
template <bool Live>
__global__ void dt_candidates(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                              const double* __restrict__ val, const uint8_t* __restrict__ keep_row,
                              const uint8_t* __restrict__ keep_col, const int32_t* __restrict__ col_nnz,
                              const double* __restrict__ AL, const double* __restrict__ AU, double zt, double tol,
                              double ratio_tol, int max_fill, const offset_t* __restrict__ tptr,
                              const int32_t* __restrict__ tidx, const double* __restrict__ tval,
                              int32_t* __restrict__ flag, int32_t* __restrict__ keep_c, int32_t* __restrict__ elim_c,
                              double* __restrict__ keep_v, double* __restrict__ elim_v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    flag[i] = 0;
    if (!keep_row[i]) continue;
    const double lhs = AL[i], rhs = AU[i];
    if (!isfinite(lhs) || !isfinite(rhs) || fabs(lhs - rhs) > tol) continue;
    int live = 0, c1 = -1, c2 = -1;
    double v1 = 0.0, v2 = 0.0;
    for (offset_t q = ptr[i]; q < ptr[i + 1] && live <= 2; ++q) {
      const int j = idx[q];
      const double a = val[q];
      if (!keep_col[j] || !(fabs(a) > zt)) continue;
      ++live;
      if (live == 1) { c1 = j; v1 = a; } else if (live == 2) { c2 = j; v2 = a; }
    }
    if (live != 2) continue;
    // _choose_doubleton_equations_columns (:170-214).
    const bool i12 = integral_ratio(v1, v2, ratio_tol), i21 = integral_ratio(v2, v1, ratio_tol);
    const int n1 = col_nnz[c1], n2 = col_nnz[c2];
    bool elim_first;
    if (n1 == 1 && n2 != 1) elim_first = true;
    else if (n1 != 1 && n2 == 1) elim_first = false;
    else if (i12 && !i21) elim_first = false;
    else if (i21 && !i12) elim_first = true;
    else elim_first = n1 < n2;
    const int e = elim_first ? c1 : c2, k = elim_first ? c2 : c1;
    const double ev = elim_first ? v1 : v2, kv = elim_first ? v2 : v1;
    // _is_acceptable_doubleton_equations_pivot (:161-168).
    if (fabs(ev) <= 0.0) continue;
    const double pr = fabs(kv / ev);
    if (!(pr <= kMaxPivotRatio && pr >= 1.0 / kMaxPivotRatio)) continue;
    if (col_nnz[e] > col_nnz[k] + max_fill + 1) continue;
    const int fill = Live ? fill_in_proxy(tptr, tidx, tval, keep_row, zt, k, e) : fill_in_proxy_stored(tptr, tidx, k, e);
    if (fill > max_fill) continue;
    flag[i] = 1;
    keep_c[i] = k; elim_c[i] = e; keep_v[i] = kv; elim_v[i] = ev;
  }
}

// The smallest flagged index (flag/pos from an exclusive scan).
__global__ void dt_scatter_first(int count, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                                 int32_t* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x)
    if (flag[q] && pos[q] == 0) out[0] = q;
}

__global__ void dt_scatter(int count, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                           const int32_t* __restrict__ ids, int32_t* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x)
    if (flag[q]) out[pos[q]] = ids ? ids[q] : q;
}

// Matching round (:989-1027): reset the owners of the active rows' columns,
// claim by atomicMin, select rows owning both columns.
__global__ void dt_reset(int k, const int32_t* __restrict__ rows, const uint8_t* __restrict__ active,
                         const int32_t* __restrict__ keep_c, const int32_t* __restrict__ elim_c,
                         int32_t* __restrict__ owner) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < k; q += gridDim.x * blockDim.x)
    if (active[q]) { const int i = rows[q]; owner[keep_c[i]] = INT_MAX; owner[elim_c[i]] = INT_MAX; }
}
__global__ void dt_claim(int k, const int32_t* __restrict__ rows, const uint8_t* __restrict__ active,
                         const uint8_t* __restrict__ blocked, const int32_t* __restrict__ keep_c,
                         const int32_t* __restrict__ elim_c, int32_t* __restrict__ owner) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < k; q += gridDim.x * blockDim.x) {
    if (!active[q]) continue;
    const int i = rows[q], kc = keep_c[i], ec = elim_c[i];
    if (!blocked[kc] && !blocked[ec]) { atomicMin(owner + kc, i); atomicMin(owner + ec, i); }
  }
}
__global__ void dt_select(int k, const int32_t* __restrict__ rows, uint8_t* __restrict__ active,
                          uint8_t* __restrict__ blocked, const int32_t* __restrict__ keep_c,
                          const int32_t* __restrict__ elim_c, const int32_t* __restrict__ owner,
                          int32_t* __restrict__ selected) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < k; q += gridDim.x * blockDim.x) {
    if (!active[q]) continue;
    const int i = rows[q], kc = keep_c[i], ec = elim_c[i];
    // A column has one owner, so no row reads a block set in this round by
    // a row it would compete with.
    if (!blocked[kc] && !blocked[ec] && owner[kc] == i && owner[ec] == i) {
      selected[q] = 1;
      active[q] = 0;
      blocked[kc] = 1;
      blocked[ec] = 1;
    }
  }
}

// _kernel_apply_doubleton_equations_batch (:1029-1117), plus the record
// captured before (:770-803) and completed after (:805-822) the update.
__global__ void dt_apply(int sel, const int32_t* __restrict__ rows, const int32_t* __restrict__ keep_c,
                         const int32_t* __restrict__ elim_c, const double* __restrict__ keep_v,
                         const double* __restrict__ elim_v, double bound_tol, double* __restrict__ l,
                         double* __restrict__ u, double* __restrict__ c, const double* __restrict__ AU,
                         uint8_t* __restrict__ keep_row, uint8_t* __restrict__ keep_col, uint8_t* __restrict__ kind,
                         double* __restrict__ alpha_out, double* __restrict__ beta_out,
                         double* __restrict__ obj_term, int32_t* __restrict__ rec_idx, double* __restrict__ rec_val,
                         int32_t* st) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < sel; t += gridDim.x * blockDim.x) {
    const int row = rows[t], k = keep_c[row], e = elim_c[row];
    const double kv = keep_v[row], ev = elim_v[row];
    const double rhs = AU[row];
    const double le = l[e], ue = u[e], lk = l[k], uk = u[k], ce = c[e], ck = c[k];
    const double alpha = -kv / ev;
    const double beta = rhs / ev;
    double ml = -INFINITY, mu = INFINITY;
    if (isfinite(le)) { const double b = (le - beta) / alpha; if (alpha > 0.0) ml = b; else mu = b; }
    if (isfinite(ue)) { const double b = (ue - beta) / alpha; if (alpha > 0.0) mu = b; else ml = b; }
    if (ml > mu) { const double tmp = ml; ml = mu; mu = tmp; }
    const double nl = isfinite(ml) ? fmax(lk, ml) : lk;
    const double nu = isfinite(mu) ? fmin(uk, mu) : uk;
    kind[t] = kPairNone;
    if (nl > nu + bound_tol) { atomicOr(st + kStInfeasible, 1); continue; }
    alpha_out[t] = alpha;
    beta_out[t] = beta;
    if (isfinite(nl) && isfinite(nu) && nu <= nl + bound_tol) {
      const double at = 0.5 * (nl + nu);
      l[k] = at;
      u[k] = at;
      keep_col[k] = 0;
      kind[t] = kPairFixed;
      obj_term[t] = ck * at;
      atomicAdd(st + kStFixed, 1);
    } else {
      l[k] = nl;
      u[k] = nu;
      c[k] = ck + ce * alpha;
      keep_row[row] = 0;
      keep_col[e] = 0;
      kind[t] = kPairSubst;
      obj_term[t] = ce * beta;
      atomicAdd(st + kStSubst, 1);
      int32_t* ri = rec_idx + 4 * int64_t(t);
      ri[0] = e; ri[1] = k; ri[2] = row; ri[3] = 0;
      double* rv = rec_val + 12 * int64_t(t);
      rv[0] = ev; rv[1] = kv; rv[2] = rhs; rv[3] = le; rv[4] = ue; rv[5] = lk; rv[6] = uk;
      rv[7] = nl; rv[8] = nu; rv[9] = ce; rv[10] = 0.0; rv[11] = 0.0;
    }
    atomicOr(st + kStAny, 1);
  }
}

__global__ void dt_subst_flags(int sel, const uint8_t* __restrict__ kind, int32_t* __restrict__ flag) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < sel; t += gridDim.x * blockDim.x)
    flag[t] = kind[t] == kPairSubst ? 1 : 0;
}

// DoubletonEquation records: indices [elim, keep, row, 0], values [a_e, a_k,
// rhs, l_e, u_e, l_k, u_k, new l_k, new u_k, c_e, 0, 0] (:641-669).
__global__ void dt_pack(int sel, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                        const int32_t* __restrict__ rec_idx, const double* __restrict__ rec_val,
                        int32_t* __restrict__ types, int64_t* __restrict__ is, int64_t* __restrict__ vs,
                        int32_t* __restrict__ oidx, double* __restrict__ oval) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < sel; t += gridDim.x * blockDim.x) {
    if (!flag[t]) continue;
    const int64_t r = pos[t];
    if (r == 0) { is[0] = 0; vs[0] = 0; }
    types[r] = 13;  // DoubletonEquation
    is[r + 1] = 4 * (r + 1);
    vs[r + 1] = 12 * (r + 1);
    for (int q = 0; q < 4; ++q) oidx[4 * r + q] = rec_idx[4 * int64_t(t) + q];
    for (int q = 0; q < 12; ++q) oval[12 * r + q] = rec_val[12 * int64_t(t) + q];
  }
}

// Columns whose entries shift row sides: eliminated columns (a * beta) and
// fixed keep columns (a * value).
__global__ void dt_roles(int sel, const int32_t* __restrict__ rows, const int32_t* __restrict__ keep_c,
                         const int32_t* __restrict__ elim_c, const uint8_t* __restrict__ kind,
                         const double* __restrict__ beta, const double* __restrict__ l, uint8_t* __restrict__ role,
                         double* __restrict__ value, int32_t* __restrict__ role_col) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < sel; t += gridDim.x * blockDim.x) {
    const int row = rows[t];
    int col = -1;
    if (kind[t] == kPairSubst) { col = elim_c[row]; value[col] = beta[t]; }
    else if (kind[t] == kPairFixed) { col = keep_c[row]; value[col] = l[col]; }
    if (col >= 0) role[col] = 1;
    role_col[t] = col;
  }
}

// Rows holding a shifting column, each listed once.
__global__ void dt_touch(int sel, const int32_t* __restrict__ role_col, const offset_t* __restrict__ tptr,
                         const int32_t* __restrict__ tidx, uint32_t* __restrict__ claimed,
                         int32_t* __restrict__ touched, int32_t* st) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < sel; w += warps) {
    const int col = role_col[w];
    if (col < 0) continue;
    for (offset_t chunk = tptr[col]; chunk < tptr[col + 1]; chunk += 32) {
      const offset_t p = chunk + lane;
      bool take = false;
      int r = 0;
      if (p < tptr[col + 1]) {
        r = tidx[p];
        const uint32_t bit = 1u << (r & 31);
        take = (atomicOr(claimed + (r >> 5), bit) & bit) == 0;
      }
      const int at = warp_append(st + kStTouched, take);
      if (take) touched[at] = r;
    }
  }
}

// Row shift of a touched kept row: its terms added in stored column order.
__global__ void dt_shift(const int32_t* __restrict__ touched, const int32_t* __restrict__ st,
                         const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                         const double* __restrict__ val, const uint8_t* __restrict__ keep_row,
                         const uint8_t* __restrict__ role, const double* __restrict__ value, double zt,
                         double* __restrict__ AL, double* __restrict__ AU) {
  const int count = st[kStTouched];
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < count; w += warps) {
    const int r = touched[w];
    if (!keep_row[r]) continue;
    double shift = 0.0;
    for (offset_t chunk = ptr[r]; chunk < ptr[r + 1]; chunk += 32) {
      const offset_t p = chunk + lane;
      double term = 0.0;
      bool has = false;
      if (p < ptr[r + 1]) {
        const int j = idx[p];
        const double a = val[p];
        if (role[j] && fabs(a) > zt) { has = true; term = a * value[j]; }
      }
      const unsigned hv = __ballot_sync(0xffffffffu, has);
      for (int k = 0; k < 32; ++k) {
        const double v = __shfl_sync(0xffffffffu, term, k);
        if (hv >> k & 1u) shift += v;
      }
    }
    if (lane == 0) { AL[r] -= shift; AU[r] -= shift; }
  }
}

// Substitution deltas alpha * a_(r, elim) at (r, keep) for kept rows r other
// than the doubleton row (:1127-1151, :1191-1229).
__global__ void dt_delta_count(int sel, const int32_t* __restrict__ rows, const int32_t* __restrict__ elim_c,
                               const uint8_t* __restrict__ kind, const offset_t* __restrict__ tptr,
                               const int32_t* __restrict__ tidx, const double* __restrict__ tval,
                               const uint8_t* __restrict__ keep_row, double zt, int32_t* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < sel; w += warps) {
    int c = 0;
    if (kind[w] == kPairSubst) {
      const int row = rows[w], e = elim_c[row];
      for (offset_t p = tptr[e] + lane; p < tptr[e + 1]; p += 32) {
        const int r = tidx[p];
        c += r != row && keep_row[r] && fabs(tval[p]) > zt ? 1 : 0;
      }
      for (int off = 16; off > 0; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off);
    }
    if (lane == 0) cnt[w] = c;
  }
}
__global__ void dt_delta_fill(int sel, const int32_t* __restrict__ rows, const int32_t* __restrict__ keep_c,
                              const int32_t* __restrict__ elim_c, const uint8_t* __restrict__ kind,
                              const double* __restrict__ alpha, const offset_t* __restrict__ tptr,
                              const int32_t* __restrict__ tidx, const double* __restrict__ tval,
                              const uint8_t* __restrict__ keep_row, double zt, const int32_t* __restrict__ pos,
                              uint64_t* __restrict__ keys, int32_t* __restrict__ order, double* __restrict__ dval) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < sel; w += warps) {
    if (kind[w] != kPairSubst) continue;
    const int row = rows[w], e = elim_c[row], k = keep_c[row];
    const double al = alpha[w];
    int64_t out = pos[w];
    for (offset_t chunk = tptr[e]; chunk < tptr[e + 1]; chunk += 32) {
      const offset_t p = chunk + lane;
      bool take = false;
      int r = 0;
      double a = 0.0;
      if (p < tptr[e + 1]) {
        r = tidx[p];
        a = tval[p];
        take = r != row && keep_row[r] && fabs(a) > zt;
      }
      const unsigned mask = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int64_t o = out + __popc(mask & ((1u << lane) - 1u));
        keys[o] = (uint64_t(uint32_t(r)) << 32) | uint32_t(k);
        order[o] = int32_t(o);
        dval[o] = al * a;
      }
      out += __popc(mask);
    }
  }
}
__global__ void dt_delta_rows(int64_t total, const uint64_t* __restrict__ keys, const int32_t* __restrict__ order,
                              const double* __restrict__ raw, int32_t* __restrict__ dcol, double* __restrict__ dv,
                              int32_t* __restrict__ row_cnt) {
  for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < total; q += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t key = keys[q];
    dcol[q] = int32_t(key & 0xffffffffu);
    dv[q] = raw[order[q]];
    atomicAdd(row_cnt + int(key >> 32), 1);
  }
}

// Merge of one row with its sorted deltas (:1242-1340), sequential: equal
// columns are summed source-first, entries with |sum| <= zero_tol dropped.
template <bool Write>
__device__ int merge_row(offset_t p, offset_t pe, const int32_t* idx, const double* val, offset_t q, offset_t qe,
                         const int32_t* dcol, const double* dv, double zt, int32_t* oidx, double* oval) {
  int cnt = 0;
  while (p < pe || q < qe) {
    const int sc = p < pe ? idx[p] : INT_MAX;
    const int dc = q < qe ? dcol[q] : INT_MAX;
    const int col = sc < dc ? sc : dc;
    double merged = 0.0;
    while (p < pe && idx[p] == col) merged += val[p++];
    while (q < qe && dcol[q] == col) merged += dv[q++];
    if (fabs(merged) > zt) {
      if (Write) { oidx[cnt] = col; oval[cnt] = merged; }
      ++cnt;
    }
  }
  return cnt;
}

// Rebuilt rows: rows without deltas of a strictly sorted matrix keep their
// entries with |a| > zero_tol (warp ballot, order kept); other rows merge
// sequentially.
template <bool Write>
__global__ void dt_rebuild(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ val, const int32_t* __restrict__ dptr,
                           const int32_t* __restrict__ dcol, const double* __restrict__ dv, double zt, bool sorted,
                           int32_t* __restrict__ cnt, const offset_t* __restrict__ optr, int32_t* __restrict__ oidx,
                           double* __restrict__ oval) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < m; r += warps) {
    const offset_t p0 = ptr[r], p1 = ptr[r + 1];
    const int q0 = dptr[r], q1 = dptr[r + 1];
    if (q0 == q1 && sorted) {
      offset_t out = Write ? optr[r] : 0;
      for (offset_t chunk = p0; chunk < p1; chunk += 32) {
        const offset_t p = chunk + lane;
        const bool keep = p < p1 && fabs(val[p]) > zt;
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (Write && keep) {
          const offset_t o = out + __popc(mask & ((1u << lane) - 1u));
          oidx[o] = idx[p];
          oval[o] = 0.0 + val[p];
        }
        out += __popc(mask);
      }
      if (!Write && lane == 0) cnt[r] = int32_t(out);
    } else if (sorted && p1 - p0 > kBlockMergeRow && q1 - q0 <= kBlockMergeDeltas) {
      continue;  // dt_rebuild_block
    } else if (lane == 0) {
      if (Write) merge_row<true>(p0, p1, idx, val, q0, q1, dcol, dv, zt, oidx + optr[r], oval + optr[r]);
      else cnt[r] = merge_row<false>(p0, p1, idx, val, q0, q1, dcol, dv, zt, nullptr, nullptr);
    }
  }
}

// Long rows with deltas (of a strictly sorted matrix): the rows the warp
// kernel leaves out, listed once.
__global__ void dt_long_delta_rows(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ dptr,
                                   int32_t* __restrict__ list, int32_t* counter) {
  const int stride = gridDim.x * blockDim.x;
  const int top = (m + stride - 1) / stride * stride;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < top; r += stride) {
    const bool take = r < m && dptr[r + 1] > dptr[r] && ptr[r + 1] - ptr[r] > kBlockMergeRow &&
                      dptr[r + 1] - dptr[r] <= kBlockMergeDeltas;
    const int at = block_append(counter, take);
    if (take) list[at] = r;
  }
}

__device__ __forceinline__ int block_exclusive_scan(int v, int* sm, int& total) {
  sm[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < kThreads; off <<= 1) {
    const int t = threadIdx.x >= unsigned(off) ? sm[threadIdx.x - off] : 0;
    __syncthreads();
    sm[threadIdx.x] += t;
    __syncthreads();
  }
  total = sm[kThreads - 1];
  const int ex = sm[threadIdx.x] - v;
  __syncthreads();
  return ex;
}

// The same merge as merge_row, one block per row: source entries are merged
// with their matching delta in parallel, the deltas without a source entry
// ("new" deltas, few) are placed by binary search, and block scans give every
// kept entry its output slot.  Valid for strictly sorted rows and sorted,
// unique delta columns.
template <bool Write>
__global__ void __launch_bounds__(kThreads)
dt_rebuild_block(const int32_t* __restrict__ list, const int32_t* __restrict__ count, const offset_t* __restrict__ ptr,
                 const int32_t* __restrict__ idx, const double* __restrict__ val, const int32_t* __restrict__ dptr,
                 const int32_t* __restrict__ dcol, const double* __restrict__ dv, double zt, int32_t* __restrict__ cnt,
                 const offset_t* __restrict__ optr, int32_t* __restrict__ oidx, double* __restrict__ oval) {
  __shared__ int scan[kThreads];
  __shared__ int kcol[kBlockMergeDeltas];
  __shared__ int kins[kBlockMergeDeltas];
  __shared__ double kval[kBlockMergeDeltas];
  const int rows = *count;
  for (int q = blockIdx.x; q < rows; q += gridDim.x) {
    const int r = list[q];
    const offset_t p0 = ptr[r];
    const int len = int(ptr[r + 1] - p0);
    const int q0 = dptr[r], nd = dptr[r + 1] - q0;
    // New deltas (no source entry in their column) that survive, in column order.
    int nk = 0;
    for (int c0 = 0; c0 < nd; c0 += kThreads) {
      const int d = c0 + threadIdx.x;
      int flag = 0, col = 0, ins = 0;
      double v = 0.0;
      if (d < nd) {
        col = dcol[q0 + d];
        int lo = 0, hi = len;
        while (lo < hi) { const int mid = (lo + hi) >> 1; if (idx[p0 + mid] < col) lo = mid + 1; else hi = mid; }
        ins = lo;
        v = 0.0 + dv[q0 + d];
        flag = (lo == len || idx[p0 + lo] != col) && fabs(v) > zt;
      }
      int total;
      const int ex = block_exclusive_scan(flag, scan, total);
      if (flag) { kcol[nk + ex] = col; kins[nk + ex] = ins; kval[nk + ex] = v; }
      nk += total;
      __syncthreads();
    }
    const offset_t base = Write ? optr[r] : 0;
    int running = 0;
    for (int c0 = 0; c0 < len; c0 += kThreads) {
      const int i = c0 + threadIdx.x;
      int keep = 0, col = 0;
      double merged = 0.0;
      if (i < len) {
        col = idx[p0 + i];
        merged = 0.0 + val[p0 + i];
        int lo = 0, hi = nd;
        while (lo < hi) { const int mid = (lo + hi) >> 1; if (dcol[q0 + mid] < col) lo = mid + 1; else hi = mid; }
        if (lo < nd && dcol[q0 + lo] == col) merged += dv[q0 + lo];
        keep = fabs(merged) > zt;
      }
      int total;
      const int ex = block_exclusive_scan(keep, scan, total);
      if (Write && i < len) {
        // New deltas inserted before source entry i: kins <= i.
        int lo = 0, hi = nk;
        while (lo < hi) { const int mid = (lo + hi) >> 1; if (kins[mid] <= i) lo = mid + 1; else hi = mid; }
        if (keep) {
          oidx[base + running + ex + lo] = col;
          oval[base + running + ex + lo] = merged;
        }
        // The new deltas that sit right before entry i.
        int first = lo;
        while (first > 0 && kins[first - 1] == i) --first;
        for (int t = first; t < lo; ++t) {
          oidx[base + running + ex + t] = kcol[t];
          oval[base + running + ex + t] = kval[t];
        }
      }
      running += total;
    }
    if (Write) {
      // New deltas after the last source entry.
      for (int t = threadIdx.x; t < nk; t += kThreads)
        if (kins[t] == len) { oidx[base + running + t] = kcol[t]; oval[base + running + t] = kval[t]; }
    } else if (threadIdx.x == 0) {
      cnt[r] = running + nk;
    }
    __syncthreads();
  }
}

// Single-row mode apply (:365-450): bounds, cost, masks and the record of
// the target row; meta = {alpha, beta, objective term}.
__global__ void dt_single_apply(const int32_t* __restrict__ acc, const int32_t* __restrict__ keep_c,
                                const int32_t* __restrict__ elim_c, const double* __restrict__ keep_v,
                                const double* __restrict__ elim_v, double bound_tol, double* __restrict__ l,
                                double* __restrict__ u, double* __restrict__ c, const double* __restrict__ AU,
                                uint8_t* __restrict__ keep_row, uint8_t* __restrict__ keep_col,
                                double* __restrict__ meta, int32_t* __restrict__ rec_idx, double* __restrict__ rec_val,
                                int32_t* st) {
  const int row = acc[0], k = keep_c[row], e = elim_c[row];
  const double kv = keep_v[row], ev = elim_v[row], rhs = AU[row];
  const double le = l[e], ue = u[e], lk = l[k], uk = u[k], ce = c[e];
  const double alpha = -kv / ev, beta = rhs / ev;
  double ml = -INFINITY, mu = INFINITY;
  if (isfinite(le)) { const double b = (le - beta) / alpha; if (alpha > 0.0) ml = b; else mu = b; }
  if (isfinite(ue)) { const double b = (ue - beta) / alpha; if (alpha > 0.0) mu = b; else ml = b; }
  if (ml > mu) { const double tmp = ml; ml = mu; mu = tmp; }
  const double nl = isfinite(ml) ? fmax(lk, ml) : lk;
  const double nu = isfinite(mu) ? fmin(uk, mu) : uk;
  if (nl > nu + bound_tol) { st[kStInfeasible] = 1; return; }
  l[k] = nl;
  u[k] = nu;
  c[k] = c[k] + ce * alpha;
  keep_row[row] = 0;
  keep_col[e] = 0;
  meta[0] = alpha;
  meta[1] = beta;
  meta[2] = ce * beta;
  rec_idx[0] = e; rec_idx[1] = k; rec_idx[2] = row; rec_idx[3] = 0;
  rec_val[0] = ev; rec_val[1] = kv; rec_val[2] = rhs; rec_val[3] = le; rec_val[4] = ue; rec_val[5] = lk;
  rec_val[6] = uk; rec_val[7] = nl; rec_val[8] = nu; rec_val[9] = ce; rec_val[10] = 0.0; rec_val[11] = 0.0;
  st[kStAny] = 1;
}

// Every row with an entry in the eliminated column shifts by a * beta (the
// first stored entry of that row, as the reference's search does).
__global__ void dt_single_shift(const int32_t* __restrict__ acc, const int32_t* __restrict__ elim_c,
                                const offset_t* __restrict__ tptr, const int32_t* __restrict__ tidx,
                                const double* __restrict__ tval, const double* __restrict__ meta,
                                const int32_t* __restrict__ st, double* __restrict__ AL, double* __restrict__ AU) {
  if (!st[kStAny]) return;
  const int e = elim_c[acc[0]];
  const offset_t b = tptr[e], end = tptr[e + 1];
  for (offset_t q = b + blockIdx.x * blockDim.x + threadIdx.x; q < end; q += offset_t(gridDim.x) * blockDim.x) {
    const int r = tidx[q];
    bool first = true;
    for (offset_t q2 = b; q2 < q && first; ++q2) first = tidx[q2] != r;
    if (!first) continue;
    const double shift = tval[q] * meta[1];
    AL[r] -= shift;
    AU[r] -= shift;
  }
}

// Single-row mode matrix (:452-500, :1814-1946): stored entries kept, the
// keep column of each row becomes a_k + alpha * a_e (inserted in column order
// when absent, dropped when |.| <= zero_tol); the target row is copied.
template <bool Write>
__global__ void dt_single_rows(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                               const double* __restrict__ val, const int32_t* __restrict__ acc,
                               const int32_t* __restrict__ keep_c, const int32_t* __restrict__ elim_c,
                               const double* __restrict__ meta, double zt, int32_t* __restrict__ cnt,
                               const offset_t* __restrict__ optr, int32_t* __restrict__ oidx,
                               double* __restrict__ oval) {
  const int target = acc[0], e = elim_c[target], k = keep_c[target];
  const double alpha = meta[0];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
    const offset_t first = ptr[r], last = ptr[r + 1];
    offset_t w = Write ? optr[r] : 0;
    if (r == target) {
      for (offset_t q = first; q < last; ++q) {
        if (Write) { oidx[w] = idx[q]; oval[w] = val[q]; }
        ++w;
      }
    } else if (first < last) {
      bool ep = false, kp = false;
      double are = 0.0, old = 0.0;
      for (offset_t q = first; q < last; ++q) {
        if (idx[q] == e) { ep = true; are = val[q]; } else if (idx[q] == k) { kp = true; old = val[q]; }
      }
      const double nk = old + alpha * are;
      const bool insert = ep && !kp && fabs(nk) > zt;
      bool inserted = !insert;
      for (offset_t q = first; q < last; ++q) {
        const int col = idx[q];
        if (insert && !inserted && col > k) {
          if (Write) { oidx[w] = k; oval[w] = nk; }
          ++w;
          inserted = true;
        }
        if (col == k) {
          if (fabs(nk) > zt) {
            if (Write) { oidx[w] = k; oval[w] = nk; }
            ++w;
          }
        } else {
          if (Write) { oidx[w] = col; oval[w] = val[q]; }
          ++w;
        }
      }
      if (insert && !inserted) {
        if (Write) { oidx[w] = k; oval[w] = nk; }
        ++w;
      }
    }
    if (!Write) cnt[r] = int32_t(w);
  }
}

int warp_grid(int64_t items) {
  return int(std::max<int64_t>(1, std::min<int64_t>((items + 7) / 8, int64_t(kNumSMs) * 16)));
}

// Single-row mode (doubleton_equations_scan = 0; rule_doubleton_equations.cu:
// 1948-2126): the smallest acceptable row (over the stored AT, unsorted as
// given) is substituted alone.
void doubleton_single_row(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  const int m = lp.m(), n = lp.n();
  if (m == 0 || n == 0) return;
  auto s = ctx().stream;
  const double zt = p.zero_tol, ratio_tol = std::fmax(1.0e-9, p.bound_tol);
  DBuf<int32_t> col_nnz(size_t(n), s), flag(size_t(m) + 1, s), pos(size_t(m) + 1, s), keep_c(size_t(m), s),
      elim_c(size_t(m), s);
  DBuf<double> keep_v(size_t(m), s), elim_v(size_t(m), s);
  GPP_LAUNCH(dt_col_nnz, grid_stride_blocks(n), kThreads, 0, s, n, lp.AT.ptr, lp.AT.idx, lp.AT.val, plan.keep_row.p,
             plan.keep_col.p, zt, col_nnz.p);
  GPP_LAUNCH(dt_candidates<false>, grid_stride_blocks(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, lp.A.val,
             plan.keep_row.p, plan.keep_col.p, col_nnz.p, plan.AL.p, plan.AU.p, zt, p.bound_tol, ratio_tol,
             p.doubleton_equations_max_fill_in_proxy, lp.AT.ptr, lp.AT.idx, lp.AT.val, flag.p, keep_c.p, elim_c.p,
             keep_v.p, elim_v.p);
  exclusive_scan_i32(flag.p, pos.p, m, s);
  if (read_scalar(pos.p + m) == 0) return;
  DBuf<int32_t> acc(size_t(1), s);
  GPP_LAUNCH(dt_scatter_first, grid_stride_blocks(m), kThreads, 0, s, m, flag.p, pos.p, acc.p);
  Status st;
  st.clear(kStWords);
  DBuf<double> meta(3, s), rec_val(12, s);
  DBuf<int32_t> rec_idx(4, s);
  GPP_LAUNCH(dt_single_apply, 1, 1, 0, s, acc.p, keep_c.p, elim_c.p, keep_v.p, elim_v.p, p.bound_tol, plan.l.p,
             plan.u.p, plan.c.p, plan.AU.p, plan.keep_row.p, plan.keep_col.p, meta.p, rec_idx.p, rec_val.p, st.d);
  GPP_LAUNCH(dt_single_shift, kNumSMs, kThreads, 0, s, acc.p, elim_c.p, lp.AT.ptr, lp.AT.idx, lp.AT.val, meta.p, st.d,
             plan.AL.p, plan.AU.p);
  const int32_t* f = st.read(kStWords);
  if (f[kStInfeasible]) { plan.has_infeasible = true; return; }
  if (p.record_postsolve_tape) {
    PostsolveSegment seg = make_segment(1, 4, 12);
    const int64_t offs[2] = {0, 4}, voffs[2] = {0, 12};
    const int32_t type = 13;  // DoubletonEquation
    check(cudaMemcpyAsync(seg.types.p, &type, sizeof(type), cudaMemcpyHostToDevice, s), "doubleton record type");
    check(cudaMemcpyAsync(seg.is.p, offs, sizeof(offs), cudaMemcpyHostToDevice, s), "doubleton record offsets");
    check(cudaMemcpyAsync(seg.vs.p, voffs, sizeof(voffs), cudaMemcpyHostToDevice, s), "doubleton record offsets");
    check(cudaMemcpyAsync(seg.idx.p, rec_idx.p, 4 * sizeof(int32_t), cudaMemcpyDeviceToDevice, s), "doubleton record");
    check(cudaMemcpyAsync(seg.val.p, rec_val.p, 12 * sizeof(double), cudaMemcpyDeviceToDevice, s), "doubleton record");
    ctx().sync("doubleton record");
    plan.tape.push_back(std::move(seg));
  }
  DBuf<int32_t> cnt(size_t(m) + 1, s);
  GPP_LAUNCH(dt_single_rows<false>, grid_stride_blocks(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, lp.A.val, acc.p,
             keep_c.p, elim_c.p, meta.p, zt, cnt.p, nullptr, nullptr, nullptr);
  DevCsr out;
  out.rows = m;
  out.cols = n;
  out.ptr = dalloc<offset_t>(size_t(m) + 1);
  exclusive_scan_i32(cnt.p, out.ptr, m, s);
  out.nnz = read_scalar(out.ptr + m);
  out.idx = dalloc<int32_t>(size_t(out.nnz));
  out.val = dalloc<double>(size_t(out.nnz));
  GPP_LAUNCH(dt_single_rows<true>, grid_stride_blocks(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, lp.A.val, acc.p,
             keep_c.p, elim_c.p, meta.p, zt, nullptr, out.ptr, out.idx, out.val);
  if (plan.has_new_A) free_csr(plan.new_A);
  plan.new_A = out;
  plan.has_new_A = true;
  plan.obj_delta += read_scalar(meta.p + 2);
  plan.has_row_action = plan.has_col_action = plan.has_change = true;
}

}  // namespace

void rule_doubleton_equations(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  if (!p.doubleton_equations_scan) { doubleton_single_row(plan, lp, p); return; }
  const int m = lp.m(), n = lp.n();
  if (m == 0 || n == 0) return;
  auto s = ctx().stream;
  const double zt = p.zero_tol, tol = p.bound_tol, ratio_tol = std::fmax(1.0e-9, p.bound_tol);

  // The fill-in proxy walks columns in ascending row order (the reference
  // sorts AT in place when it is not, rule_doubleton_equations.cu:126-148).
  DevCsr sorted_at;
  const bool at_sorted = lp.AT_sorted();
  if (!at_sorted) sorted_at = transpose_csr(lp.A, s);
  const DevCsr& AT = at_sorted ? lp.AT : sorted_at;
  struct Release {
    DevCsr& M;
    bool own;
    ~Release() { if (own) free_csr(M); }
  } release{sorted_at, !at_sorted};

  DBuf<int32_t> col_nnz(size_t(n), s), flag(size_t(m) + 1, s), pos(size_t(m) + 1, s), keep_c(size_t(m), s),
      elim_c(size_t(m), s);
  DBuf<double> keep_v(size_t(m), s), elim_v(size_t(m), s);
  GPP_LAUNCH(dt_col_nnz, grid_stride_blocks(n), kThreads, 0, s, n, AT.ptr, AT.idx, AT.val, plan.keep_row.p,
             plan.keep_col.p, zt, col_nnz.p);
  GPP_LAUNCH(dt_candidates<true>, grid_stride_blocks(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, lp.A.val,
             plan.keep_row.p, plan.keep_col.p, col_nnz.p, plan.AL.p, plan.AU.p, zt, tol, ratio_tol,
             p.doubleton_equations_max_fill_in_proxy, AT.ptr, AT.idx, AT.val, flag.p, keep_c.p, elim_c.p, keep_v.p,
             elim_v.p);
  exclusive_scan_i32(flag.p, pos.p, m, s);
  const int acceptable = read_scalar(pos.p + m);
  if (acceptable == 0) return;
  DBuf<int32_t> acc(size_t(acceptable), s);
  GPP_LAUNCH(dt_scatter, grid_stride_blocks(m), kThreads, 0, s, m, flag.p, pos.p, nullptr, acc.p);

  // Matching rounds over the acceptable rows (ascending).
  DBuf<uint8_t> active(size_t(acceptable), s), blocked(size_t(n), s);
  DBuf<int32_t> owner(size_t(n), s), chosen(size_t(acceptable) + 1, s), cpos(size_t(acceptable) + 1, s);
  check(cudaMemsetAsync(active.p, 1, size_t(acceptable), s), "doubleton active");
  blocked.zero();
  chosen.zero();
  const int gk = grid_stride_blocks(acceptable);
  for (int round = 0; round < kRounds; ++round) {
    GPP_LAUNCH(dt_reset, gk, kThreads, 0, s, acceptable, acc.p, active.p, keep_c.p, elim_c.p, owner.p);
    GPP_LAUNCH(dt_claim, gk, kThreads, 0, s, acceptable, acc.p, active.p, blocked.p, keep_c.p, elim_c.p, owner.p);
    GPP_LAUNCH(dt_select, gk, kThreads, 0, s, acceptable, acc.p, active.p, blocked.p, keep_c.p, elim_c.p, owner.p,
               chosen.p);
  }
  exclusive_scan_i32(chosen.p, cpos.p, acceptable, s);
  const int sel = read_scalar(cpos.p + acceptable);
  const double ratio = double(sel) / double(acceptable);
  if (sel == 0 || sel < p.doubleton_equations_min_selected_per_batch || ratio < p.doubleton_equations_min_selected_ratio)
    return;
  DBuf<int32_t> rows(size_t(sel), s);
  GPP_LAUNCH(dt_scatter, gk, kThreads, 0, s, acceptable, chosen.p, cpos.p, acc.p, rows.p);

  // Apply against the values before the batch (columns are distinct).
  Status st;
  st.clear(kStWords);
  DBuf<uint8_t> kind(size_t(sel), s);
  DBuf<double> alpha(size_t(sel), s), beta(size_t(sel), s), obj_term(size_t(sel), s), rec_val(size_t(sel) * 12, s);
  DBuf<int32_t> rec_idx(size_t(sel) * 4, s);
  const int gs = grid_stride_blocks(sel);
  GPP_LAUNCH(dt_apply, gs, kThreads, 0, s, sel, rows.p, keep_c.p, elim_c.p, keep_v.p, elim_v.p, p.bound_tol,
             plan.l.p, plan.u.p, plan.c.p, plan.AU.p, plan.keep_row.p, plan.keep_col.p, kind.p, alpha.p, beta.p,
             obj_term.p, rec_idx.p, rec_val.p, st.d);
  const int32_t* f = st.read(kStWords);
  if (f[kStInfeasible]) { plan.has_infeasible = true; return; }
  if (!f[kStAny]) return;
  const int subst = f[kStSubst];

  DBuf<int32_t> sflag(size_t(sel) + 1, s), spos(size_t(sel) + 1, s);
  if (subst) {
    GPP_LAUNCH(dt_subst_flags, gs, kThreads, 0, s, sel, kind.p, sflag.p);
    exclusive_scan_i32(sflag.p, spos.p, sel, s);
    if (p.record_postsolve_tape) {
      PostsolveSegment seg = make_segment(subst, 4 * int64_t(subst), 12 * int64_t(subst));
      GPP_LAUNCH(dt_pack, gs, kThreads, 0, s, sel, sflag.p, spos.p, rec_idx.p, rec_val.p, seg.types.p, seg.is.p,
                 seg.vs.p, seg.idx.p, seg.val.p);
      plan.tape.push_back(std::move(seg));
    }
  }

  // Row shifts.
  {
    DBuf<uint8_t> role(size_t(n), s);
    DBuf<double> value(size_t(n), s);
    DBuf<int32_t> role_col(size_t(sel), s), touched(size_t(m), s);
    DBuf<uint32_t> claimed(size_t(m + 31) / 32, s);
    role.zero();
    claimed.zero();
    GPP_LAUNCH(dt_roles, gs, kThreads, 0, s, sel, rows.p, keep_c.p, elim_c.p, kind.p, beta.p, plan.l.p, role.p,
               value.p, role_col.p);
    GPP_LAUNCH(dt_touch, warp_grid(sel), kThreads, 0, s, sel, role_col.p, AT.ptr, AT.idx, claimed.p, touched.p, st.d);
    const int ntouched = st.read(kStWords)[kStTouched];
    if (ntouched)
      GPP_LAUNCH(dt_shift, warp_grid(ntouched), kThreads, 0, s, touched.p, st.d, lp.A.ptr, lp.A.idx, lp.A.val,
                 plan.keep_row.p, role.p, value.p, zt, plan.AL.p, plan.AU.p);
  }

  // Rebuilt matrix.
  if (subst) {
    DBuf<int32_t> dcnt(size_t(sel) + 1, s), dpos(size_t(sel) + 1, s);
    GPP_LAUNCH(dt_delta_count, warp_grid(sel), kThreads, 0, s, sel, rows.p, elim_c.p, kind.p, AT.ptr, AT.idx, AT.val,
               plan.keep_row.p, zt, dcnt.p);
    exclusive_scan_i32(dcnt.p, dpos.p, sel, s);
    const int total = read_scalar(dpos.p + sel);
    DBuf<uint64_t> keys(size_t(std::max(total, 1)), s);
    DBuf<int32_t> order(size_t(std::max(total, 1)), s), dcol(size_t(std::max(total, 1)), s),
        row_cnt(size_t(m) + 1, s), dptr(size_t(m) + 1, s);
    DBuf<double> raw(size_t(std::max(total, 1)), s), dv(size_t(std::max(total, 1)), s);
    row_cnt.zero();
    if (total) {
      GPP_LAUNCH(dt_delta_fill, warp_grid(sel), kThreads, 0, s, sel, rows.p, keep_c.p, elim_c.p, kind.p, alpha.p,
                 AT.ptr, AT.idx, AT.val, plan.keep_row.p, zt, dpos.p, keys.p, order.p, raw.p);
      radix_sort_pairs(keys.p, order.p, total, s);
      GPP_LAUNCH(dt_delta_rows, grid_stride_blocks(total), kThreads, 0, s, int64_t(total), keys.p, order.p, raw.p,
                 dcol.p, dv.p, row_cnt.p);
    }
    exclusive_scan_i32(row_cnt.p, dptr.p, m, s);
    const bool a_sorted = lp.A_sorted();
    DBuf<int32_t> cnt(size_t(m) + 1, s), long_rows(size_t(m), s), long_count(1, s);
    long_count.zero();
    if (a_sorted)
      GPP_LAUNCH(dt_long_delta_rows, grid_stride_blocks(m), kThreads, 0, s, m, lp.A.ptr, dptr.p, long_rows.p,
                 long_count.p);
    GPP_LAUNCH(dt_rebuild<false>, warp_grid(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, lp.A.val, dptr.p, dcol.p,
               dv.p, zt, a_sorted, cnt.p, nullptr, nullptr, nullptr);
    if (a_sorted)
      GPP_LAUNCH(dt_rebuild_block<false>, kNumSMs * 4, kThreads, 0, s, long_rows.p, long_count.p, lp.A.ptr, lp.A.idx,
                 lp.A.val, dptr.p, dcol.p, dv.p, zt, cnt.p, nullptr, nullptr, nullptr);
    DevCsr out;
    out.rows = m;
    out.cols = n;
    out.ptr = dalloc<offset_t>(size_t(m) + 1);
    exclusive_scan_i32(cnt.p, out.ptr, m, s);
    out.nnz = read_scalar(out.ptr + m);
    out.idx = dalloc<int32_t>(size_t(out.nnz));
    out.val = dalloc<double>(size_t(out.nnz));
    GPP_LAUNCH(dt_rebuild<true>, warp_grid(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, lp.A.val, dptr.p, dcol.p,
               dv.p, zt, a_sorted, nullptr, out.ptr, out.idx, out.val);
    if (a_sorted)
      GPP_LAUNCH(dt_rebuild_block<true>, kNumSMs * 4, kThreads, 0, s, long_rows.p, long_count.p, lp.A.ptr, lp.A.idx,
                 lp.A.val, dptr.p, dcol.p, dv.p, zt, nullptr, out.ptr, out.idx, out.val);
    if (plan.has_new_A) free_csr(plan.new_A);
    plan.new_A = out;
    plan.has_new_A = true;
  }

  // Objective: substitution terms, then fixed terms, each in batch order.
  const auto [hk, ho] = to_host2(kind.p, size_t(sel), obj_term.p, size_t(sel));
  double obj = 0.0, fixed_obj = 0.0;
  for (int t = 0; t < sel; ++t) {
    if (hk[size_t(t)] == kPairSubst) obj += ho[size_t(t)];
    else if (hk[size_t(t)] == kPairFixed) fixed_obj += ho[size_t(t)];
  }
  plan.obj_delta += obj;
  plan.obj_delta += fixed_obj;
  plan.has_row_action = subst > 0;
  plan.has_col_action = true;
  plan.has_change = true;
}

}  // namespace gpp
