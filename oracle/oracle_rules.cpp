// Oracle presolve rules: CPU restatements of the reference's apply_rule_*
// functions.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include "oracle_rules.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <stdexcept>

namespace oracle {

namespace {
inline bool fin(double x) { return std::isfinite(x); }
// Order-free max / min of candidate bounds, as the engine's 64-bit integer
// reductions combine them: the reference's load-and-CAS loop
// (rule_bound_strengthening.cu:299-335) for every input except the tie
// +0 / -0, which the loop resolves by arrival order; here max keeps +0 and
// min keeps -0.
inline void max_into(double& cur, double v) {
  if (v > cur || (v == 0.0 && cur == 0.0 && std::signbit(cur) && !std::signbit(v))) cur = v;
}
inline void min_into(double& cur, double v) {
  if (v < cur || (v == 0.0 && cur == 0.0 && !std::signbit(cur) && std::signbit(v))) cur = v;
}
}

void refresh_stats(Stats& s, const Lp& lp, const Plan& plan) {
  // refresh_live_stats (gpu_presolve_kernels.cu:493-517): rows over A with
  // keep_row outer / keep_col inner, columns over AT with the roles swapped.
  const int m = lp.m(), n = lp.n();
  s.row_nnz.assign(m, 0); s.empty_row.assign(m, 0); s.singleton_row.assign(m, 0);
  s.srow_col.assign(m, -1); s.srow_val.assign(m, 0.0);
  s.col_nnz.assign(n, 0); s.empty_col.assign(n, 0); s.singleton_col.assign(n, 0);
  s.scol_row.assign(n, -1); s.scol_val.assign(n, 0.0);
  s.live_nnz = 0;
  live_stats(lp.A, plan.keep_row.data(), plan.keep_col.data(), s.row_nnz.data(), s.empty_row.data(),
             s.singleton_row.data(), s.srow_col.data(), s.srow_val.data(), &s.live_nnz);
  live_stats(lp.AT, plan.keep_col.data(), plan.keep_row.data(), s.col_nnz.data(), s.empty_col.data(),
             s.singleton_col.data(), s.scol_row.data(), s.scol_val.data(), nullptr);
}

// Row sums of a_ij * v_j over kept rows and selected columns, in ascending
// column order (the reference accumulates the same terms with atomicAdd).
static std::vector<double> row_shift_gather(const Lp& lp, const std::vector<uint8_t>& keep_row,
                                            const std::vector<uint8_t>& selected,
                                            const std::vector<double>& value, bool absolute,
                                            const std::vector<double>* radius = nullptr) {
  std::vector<double> shift(lp.m(), 0.0);
  for (int i = 0; i < lp.m(); ++i) {
    if (!keep_row[i]) continue;
    double acc = 0.0;
    for (int p = lp.A.ptr[i]; p < lp.A.ptr[i + 1]; ++p) {
      const int j = lp.A.idx[p];
      if (!selected[j]) continue;
      if (absolute) {
        if ((*radius)[j] > 0.0) acc += std::fabs(lp.A.val[p]) * (*radius)[j];
      } else {
        acc += lp.A.val[p] * value[j];
      }
    }
    shift[i] = acc;
  }
  return shift;
}

static double domain_objective(const std::vector<double>& contrib, const Plan& plan) {
  // sum_cleanup_domain (cleanup_support.cuh:13-31) restricted to the rule's
  // entry domain; nonselected entries are zero, so the canonical sum over the
  // compacted domain equals the sum over the masked full vector.
  std::vector<double> v(contrib);
  if (plan.rule_entry_keep_col)
    for (size_t j = 0; j < v.size(); ++j)
      if (!(*plan.rule_entry_keep_col)[j]) v[j] = 0.0;
  return det_sum(v);
}

void rule_fixed_variables(Plan& plan, const Lp& lp, const gpp_params& p) {
  // apply_rule_infeasible_and_fixed_variables (rule_infeasible_and_fixed_variables.cu:65-348).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int n = lp.n(), m = lp.m();
  if (n == 0) return;
  std::vector<uint8_t> fixed(n, 0);
  std::vector<double> fval(n, 0.0), contrib(n, 0.0), radius(n, 0.0);
  for (int j = 0; j < n; ++j) {
    if (!plan.keep_col[j]) continue;
    const double lj = plan.l[j], uj = plan.u[j];
    if (fin(lj) && fin(uj) && lj <= uj && uj - lj <= p.bound_tol) {
      const double vj = lj + 0.5 * (uj - lj);
      radius[j] = std::fmax(vj - lj, uj - vj);
      fixed[j] = 1;
      fval[j] = vj;
      contrib[j] = plan.c[j] * vj;
    }
  }
  // Row error budget (sum of |a| * radius over candidates) and the filter.
  const std::vector<double> row_error = row_shift_gather(lp, plan.keep_row, fixed, fval, true, &radius);
  const double budget = 0.1 * p.feasibility_tol;
  for (int j = 0; j < n; ++j) {
    if (!fixed[j] || plan.l[j] == plan.u[j]) continue;
    for (int q = lp.AT.ptr[j]; q < lp.AT.ptr[j + 1]; ++q) {
      const int row = lp.AT.idx[q];
      if (plan.keep_row[row] && !(row_error[row] <= budget)) {
        fixed[j] = 0;
        contrib[j] = 0.0;
        break;
      }
    }
  }
  int count = 0;
  for (int j = 0; j < n; ++j) count += fixed[j];
  if (count == 0) return;
  const std::vector<double> shift = row_shift_gather(lp, plan.keep_row, fixed, fval, false);
  for (int j = 0; j < n; ++j)
    if (fixed[j]) { plan.l[j] = fval[j]; plan.u[j] = fval[j]; plan.keep_col[j] = 0; }
  for (int i = 0; i < m; ++i) { plan.AL[i] -= shift[i]; plan.AU[i] -= shift[i]; }
  plan.obj_delta += domain_objective(contrib, plan);
  plan.has_col_action = true;
  plan.has_change = true;
}

void rule_empty_columns(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p) {
  // apply_rule_empty_columns (empty_rows_and_columns/columns.cu:64-249).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int n = lp.n();
  if (n == 0) return;
  bool infeasible = false, unbounded = false, any = false;
  std::vector<uint8_t> fixed(n, 0);
  std::vector<double> fval(n, 0.0), contrib(n, 0.0);
  for (int j = 0; j < n; ++j) {
    if (!(plan.keep_col[j] && s.empty_col[j])) continue;
    const double cj = plan.c[j], lj = plan.l[j], uj = plan.u[j];
    if (lj > uj + p.bound_tol) { infeasible = true; continue; }
    if ((cj > p.zero_tol && !fin(lj)) || (cj < -p.zero_tol && !fin(uj))) { unbounded = true; continue; }
    double v = 0.0;
    if (cj > p.zero_tol) v = lj;
    else if (cj < -p.zero_tol) v = uj;
    else if (fin(lj)) v = lj;
    else if (fin(uj)) v = uj;
    fixed[j] = 1; fval[j] = v; contrib[j] = cj * v; any = true;
  }
  if (infeasible) { plan.has_infeasible = true; return; }
  if (unbounded) { plan.has_unbounded = true; return; }
  if (!any) return;
  for (int j = 0; j < n; ++j)
    if (fixed[j]) { plan.l[j] = fval[j]; plan.u[j] = fval[j]; plan.keep_col[j] = 0; }
  plan.obj_delta += domain_objective(contrib, plan);
  plan.has_col_action = true;
  plan.has_change = true;
}

void rule_empty_rows(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p) {
  // apply_rule_empty_rows (empty_rows_and_columns/rows.cu:26-121).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m();
  if (m == 0) return;
  bool infeasible = false, any = false;
  const double tol = p.feasibility_tol;
  for (int i = 0; i < m; ++i) {
    if (!(plan.keep_row[i] && s.row_nnz[i] == 0)) continue;
    if (plan.AL[i] <= tol && plan.AU[i] >= -tol) any = true; else infeasible = true;
  }
  if (infeasible) { plan.has_infeasible = true; return; }
  if (!any) return;
  for (int i = 0; i < m; ++i)
    if (plan.keep_row[i] && s.row_nnz[i] == 0 && plan.AL[i] <= tol && plan.AU[i] >= -tol)
      plan.keep_row[i] = 0;
  plan.has_row_action = plan.has_row_deletion = plan.has_change = true;
}

void rule_singleton_rows(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p) {
  // apply_rule_singleton_rows (rule_singleton_rows.cu:76-275).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (m == 0) return;
  std::vector<double> cl(plan.l), cu(plan.u);
  std::vector<uint8_t> remove(m, 0);
  bool any_remove = false;
  for (int i = 0; i < m; ++i) {
    if (!(plan.keep_row[i] && s.singleton_row[i])) continue;
    const int col = s.srow_col[i];
    const double a = s.srow_val[i];
    if (col < 0 || col >= n || !(std::fabs(a) > p.zero_tol)) continue;
    const double lo = plan.AL[i], hi = plan.AU[i];
    const double il = a > 0.0 ? lo / a : hi / a;
    const double iu = a > 0.0 ? hi / a : lo / a;
    max_into(cl[col], il);   // atomic_max_double
    min_into(cu[col], iu);   // atomic_min_double
    remove[i] = 1;
    any_remove = true;
  }
  bool infeasible = false, bounds_changed = false;
  for (int j = 0; j < n; ++j) {
    if (cl[j] > cu[j] + p.bound_tol) infeasible = true;
    if (cl[j] != plan.l[j] || cu[j] != plan.u[j]) bounds_changed = true;
  }
  if (infeasible) { plan.has_infeasible = true; return; }
  if (!any_remove && !bounds_changed) return;
  for (int i = 0; i < m; ++i) if (remove[i]) plan.keep_row[i] = 0;
  plan.l = cl;
  plan.u = cu;
  plan.has_row_action = true;
  plan.has_row_deletion = plan.has_row_deletion || any_remove;
  plan.has_change = true;
}

// ---- doubleton equations ----------------------------------------------------

namespace {
constexpr int kDoubletonRounds = 8;          // DOUBLETON_EQUATION_BATCH_MATCHING_ROUNDS
constexpr double kDoubletonMaxPivotRatio = 1.0e3;

bool integral_ratio(double num, double den, double tol) {
  // _is_integral_ratio_doubleton_equations (rule_doubleton_equations.cu:150-159).
  if (std::fabs(den) <= tol) return false;
  const double r = std::fabs(num / den);
  if (!std::isfinite(r)) return false;
  return std::fabs(r - std::nearbyint(r)) <= tol;
}

bool strictly_sorted(const Csr& M) {
  for (int r = 0; r < M.rows; ++r)
    for (int p = M.ptr[r] + 1; p < M.ptr[r + 1]; ++p)
      if (M.idx[p - 1] >= M.idx[p]) return false;
  return true;
}

// _doubleton_equations_fill_in_proxy_device_live (rule_doubleton_equations.cu:843-890).
int fill_in_proxy(const Csr& AT, const std::vector<uint8_t>& keep_row, double zt, int keep, int elim) {
  int fill = -1;
  int jj = AT.ptr[keep], kk = AT.ptr[elim];
  const int js = AT.ptr[keep + 1], ks = AT.ptr[elim + 1];
  if (js <= jj || ks <= kk) return fill;
  auto next_live = [&](int col, int& pos) {
    while (pos < AT.ptr[col + 1]) {
      const int r = AT.idx[pos];
      if (keep_row[r] && std::fabs(AT.val[pos]) > zt) return r;
      ++pos;
    }
    return INT_MAX;
  };
  while (jj < js && kk < ks) {
    int jl = jj, kl = kk;
    const int rj = next_live(keep, jl), rk = next_live(elim, kl);
    if (rj == INT_MAX || rk == INT_MAX) break;
    if (rj == rk) { jj = jl + 1; kk = kl + 1; }
    else if (rk < rj) { kk = kl + 1; ++fill; }
    else jj = jl + 1;
  }
  while (kk < ks) {
    int kl = kk;
    if (next_live(elim, kl) == INT_MAX) break;
    ++fill;
    kk = kl + 1;
  }
  return fill;
}
}  // namespace

namespace {
// _doubleton_equations_fill_in_proxy_device (rule_doubleton_equations.cu:216-243):
// over the stored entries of AT, masks ignored.
int fill_in_proxy_stored(const Csr& AT, int keep, int elim) {
  int fill = -1;
  int jj = AT.ptr[keep], kk = AT.ptr[elim];
  const int js = AT.ptr[keep + 1], ks = AT.ptr[elim + 1];
  if (js <= jj || ks <= kk) return fill;
  while (jj < js && kk < ks) {
    const int kr = AT.idx[jj], er = AT.idx[kk];
    if (kr == er) { ++jj; ++kk; }
    else if (er < kr) { ++kk; ++fill; }
    else ++jj;
  }
  return fill + (ks - kk);
}

// Single-row mode (doubleton_equations_scan = 0; rule_doubleton_equations.cu:
// 273-512, 1814-2126): the smallest acceptable row is substituted; every row
// side shifts by a_(r,elim) * beta, and the matrix keeps its stored entries
// except the keep column, which becomes a_(r,keep) + alpha * a_(r,elim).
void doubleton_single_row(Plan& plan, const Lp& lp, const gpp_params& p) {
  const int m = lp.m(), n = lp.n();
  if (m == 0 || n == 0) return;
  const Csr& A = lp.A;
  const double zt = p.zero_tol, tol = p.bound_tol, ratio_tol = std::fmax(1.0e-9, p.bound_tol);
  std::vector<int> col_nnz(size_t(n), 0);
  for (int j = 0; j < n; ++j) {
    if (!plan.keep_col[j]) continue;
    for (int q = lp.AT.ptr[j]; q < lp.AT.ptr[j + 1]; ++q)
      if (plan.keep_row[lp.AT.idx[q]] && std::fabs(lp.AT.val[q]) > zt) ++col_nnz[j];
  }
  int target = -1, e = -1, k = -1;
  double ev = 0.0, kv = 0.0;
  for (int i = 0; i < m && target < 0; ++i) {
    if (!plan.keep_row[i]) continue;
    const double lhs = plan.AL[i], rhs = plan.AU[i];
    if (!fin(lhs) || !fin(rhs) || std::fabs(lhs - rhs) > tol) continue;
    int live = 0, c1 = -1, c2 = -1;
    double v1 = 0.0, v2 = 0.0;
    for (int q = A.ptr[i]; q < A.ptr[i + 1] && live <= 2; ++q) {
      const int j = A.idx[q];
      if (!plan.keep_col[j] || !(std::fabs(A.val[q]) > zt)) continue;
      ++live;
      if (live == 1) { c1 = j; v1 = A.val[q]; } else if (live == 2) { c2 = j; v2 = A.val[q]; }
    }
    if (live != 2) continue;
    const bool i12 = integral_ratio(v1, v2, ratio_tol), i21 = integral_ratio(v2, v1, ratio_tol);
    bool elim_first;
    if (col_nnz[c1] == 1 && col_nnz[c2] != 1) elim_first = true;
    else if (col_nnz[c1] != 1 && col_nnz[c2] == 1) elim_first = false;
    else if (i12 && !i21) elim_first = false;
    else if (i21 && !i12) elim_first = true;
    else elim_first = col_nnz[c1] < col_nnz[c2];
    const int ce = elim_first ? c1 : c2, ck = elim_first ? c2 : c1;
    const double cev = elim_first ? v1 : v2, ckv = elim_first ? v2 : v1;
    if (std::fabs(cev) <= 0.0) continue;
    const double pr = std::fabs(ckv / cev);
    if (!(pr <= kDoubletonMaxPivotRatio && pr >= 1.0 / kDoubletonMaxPivotRatio)) continue;
    if (col_nnz[ce] > col_nnz[ck] + p.doubleton_equations_max_fill_in_proxy + 1) continue;
    if (fill_in_proxy_stored(lp.AT, ck, ce) > p.doubleton_equations_max_fill_in_proxy) continue;
    target = i; e = ce; k = ck; ev = cev; kv = ckv;
  }
  if (target < 0) return;
  const double rhs = plan.AU[target];
  const double le = plan.l[e], ue = plan.u[e], lk = plan.l[k], uk = plan.u[k], ce = plan.c[e];
  const double alpha = -kv / ev, beta = rhs / ev;
  double ml = -INFINITY, mu = INFINITY;
  if (fin(le)) { const double b = (le - beta) / alpha; if (alpha > 0.0) ml = b; else mu = b; }
  if (fin(ue)) { const double b = (ue - beta) / alpha; if (alpha > 0.0) mu = b; else ml = b; }
  if (ml > mu) std::swap(ml, mu);
  const double nl = fin(ml) ? std::fmax(lk, ml) : lk;
  const double nu = fin(mu) ? std::fmin(uk, mu) : uk;
  if (nl > nu + p.bound_tol) { plan.has_infeasible = true; return; }
  for (int q = lp.AT.ptr[e]; q < lp.AT.ptr[e + 1]; ++q) {
    const int r = lp.AT.idx[q];
    bool first = true;
    for (int q2 = lp.AT.ptr[e]; q2 < q; ++q2) first = first && lp.AT.idx[q2] != r;
    if (!first) continue;
    const double shift = lp.AT.val[q] * beta;
    plan.AL[r] -= shift;
    plan.AU[r] -= shift;
  }
  plan.l[k] = nl;
  plan.u[k] = nu;
  plan.c[k] += ce * alpha;
  plan.keep_row[target] = 0;
  plan.keep_col[e] = 0;
  if (p.record_postsolve_tape)
    plan.tape.add(DoubletonEquation, {e, k, target, 0}, {ev, kv, rhs, le, ue, lk, uk, nl, nu, ce, 0.0, 0.0});
  Csr out;
  out.rows = m;
  out.cols = n;
  out.ptr.assign(size_t(m) + 1, 0);
  for (int r = 0; r < m; ++r) {
    const int first = A.ptr[r], last = A.ptr[r + 1];
    if (r == target) {
      for (int q = first; q < last; ++q) { out.idx.push_back(A.idx[q]); out.val.push_back(A.val[q]); }
    } else if (first < last) {
      bool ep = false, kp = false;
      double are = 0.0, old = 0.0;
      for (int q = first; q < last; ++q) {
        if (A.idx[q] == e) { ep = true; are = A.val[q]; } else if (A.idx[q] == k) { kp = true; old = A.val[q]; }
      }
      const double nk = old + alpha * are;
      const bool insert = ep && !kp && std::fabs(nk) > zt;
      bool inserted = !insert;
      for (int q = first; q < last; ++q) {
        const int col = A.idx[q];
        if (insert && !inserted && col > k) { out.idx.push_back(k); out.val.push_back(nk); inserted = true; }
        if (col == k) {
          if (std::fabs(nk) > zt) { out.idx.push_back(k); out.val.push_back(nk); }
        } else {
          out.idx.push_back(col);
          out.val.push_back(A.val[q]);
        }
      }
      if (insert && !inserted) { out.idx.push_back(k); out.val.push_back(nk); }
    }
    out.ptr[size_t(r) + 1] = int(out.idx.size());
  }
  plan.new_A = std::move(out);
  plan.has_new_A = true;
  plan.obj_delta += ce * beta;
  plan.has_row_action = plan.has_col_action = plan.has_change = true;
}
}  // namespace

void rule_doubleton_equations(Plan& plan, const Lp& lp, const gpp_params& p) {
  // apply_rule_doubleton_equations -> _batch -> _batch_once
  // (rule_doubleton_equations.cu:1512-1812, 1948-1957): one batch of
  // non-overlapping doubleton equalities per call.
  if (plan.has_infeasible || plan.has_unbounded) return;
  if (!p.doubleton_equations_scan) { doubleton_single_row(plan, lp, p); return; }
  const int m = lp.m(), n = lp.n();
  if (m == 0 || n == 0) return;
  const Csr& A = lp.A;
  const Csr ATs = strictly_sorted(lp.AT) ? lp.AT : transpose(lp.A);
  const double zt = p.zero_tol, tol = p.bound_tol, ratio_tol = std::fmax(1.0e-9, p.bound_tol);

  // _kernel_doubleton_equations_live_col_nnz (:245-271).
  std::vector<int> col_nnz(size_t(n), 0);
  for (int j = 0; j < n; ++j) {
    if (!plan.keep_col[j]) continue;
    int cnt = 0;
    for (int q = ATs.ptr[j]; q < ATs.ptr[j + 1]; ++q)
      if (plan.keep_row[ATs.idx[q]] && std::fabs(ATs.val[q]) > zt) ++cnt;
    col_nnz[j] = cnt;
  }
  // Candidates (:892-958) and fill-in acceptance (:960-987).
  std::vector<uint8_t> active(size_t(m), 0);
  std::vector<int> ke(size_t(m), -1), el(size_t(m), -1);
  std::vector<double> kv(size_t(m), 0.0), ev(size_t(m), 0.0);
  int acceptable = 0;
  for (int i = 0; i < m; ++i) {
    if (!plan.keep_row[i]) continue;
    const double lhs = plan.AL[i], rhs = plan.AU[i];
    if (!fin(lhs) || !fin(rhs) || std::fabs(lhs - rhs) > tol) continue;
    int live = 0, c1 = -1, c2 = -1;
    double v1 = 0.0, v2 = 0.0;
    for (int q = A.ptr[i]; q < A.ptr[i + 1] && live <= 2; ++q) {
      const int j = A.idx[q];
      if (!plan.keep_col[j] || !(std::fabs(A.val[q]) > zt)) continue;
      ++live;
      if (live == 1) { c1 = j; v1 = A.val[q]; } else if (live == 2) { c2 = j; v2 = A.val[q]; }
    }
    if (live != 2) continue;
    // _choose_doubleton_equations_columns (:170-214).
    const bool i12 = integral_ratio(v1, v2, ratio_tol), i21 = integral_ratio(v2, v1, ratio_tol);
    bool elim_first;
    if (col_nnz[c1] == 1 && col_nnz[c2] != 1) elim_first = true;
    else if (col_nnz[c1] != 1 && col_nnz[c2] == 1) elim_first = false;
    else if (i12 && !i21) elim_first = false;
    else if (i21 && !i12) elim_first = true;
    else elim_first = col_nnz[c1] < col_nnz[c2];
    const int e = elim_first ? c1 : c2, k = elim_first ? c2 : c1;
    const double evl = elim_first ? v1 : v2, kvl = elim_first ? v2 : v1;
    // _is_acceptable_doubleton_equations_pivot (:161-168).
    if (std::fabs(evl) <= 0.0) continue;
    const double pr = std::fabs(kvl / evl);
    if (!(pr <= kDoubletonMaxPivotRatio && pr >= 1.0 / kDoubletonMaxPivotRatio)) continue;
    if (col_nnz[e] > col_nnz[k] + p.doubleton_equations_max_fill_in_proxy + 1) continue;
    if (fill_in_proxy(ATs, plan.keep_row, zt, k, e) > p.doubleton_equations_max_fill_in_proxy) continue;
    active[i] = 1;
    ke[i] = k; el[i] = e; kv[i] = kvl; ev[i] = evl;
    ++acceptable;
  }
  // Matching rounds (:989-1027, :1604-1613): each round, a row that owns both
  // of its unblocked columns (the smallest claiming row) is selected.
  std::vector<uint8_t> blocked(size_t(n), 0), selected(size_t(m), 0);
  for (int round = 0; round < kDoubletonRounds; ++round) {
    std::vector<int> owner(size_t(n), INT_MAX);
    for (int i = 0; i < m; ++i)
      if (active[i] && !blocked[ke[i]] && !blocked[el[i]]) {
        owner[ke[i]] = std::min(owner[ke[i]], i);
        owner[el[i]] = std::min(owner[el[i]], i);
      }
    std::vector<int> won;
    for (int i = 0; i < m; ++i)
      if (active[i] && !blocked[ke[i]] && !blocked[el[i]] && owner[ke[i]] == i && owner[el[i]] == i) won.push_back(i);
    for (int i : won) { selected[i] = 1; active[i] = 0; blocked[ke[i]] = blocked[el[i]] = 1; }
  }
  std::vector<int> rows;
  for (int i = 0; i < m; ++i) if (selected[i]) rows.push_back(i);
  const int sel = int(rows.size());
  const double ratio = acceptable == 0 ? 0.0 : double(sel) / double(acceptable);
  if (sel == 0 || sel < p.doubleton_equations_min_selected_per_batch || ratio < p.doubleton_equations_min_selected_ratio)
    return;

  // Apply (:1029-1117) against the values before the batch; keep and
  // eliminated columns are distinct across the batch.
  struct Rec { int e, k, row; double ev, kv, au, el, eu, kl, ku, nkl, nku, ec; };
  std::vector<Rec> recs;
  std::vector<uint8_t> subst(size_t(sel), 0), fixed(size_t(sel), 0);
  std::vector<double> beta_of(size_t(sel), 0.0), alpha_of(size_t(sel), 0.0);
  bool infeasible = false, any = false;
  double obj = 0.0, fixed_obj = 0.0;
  for (int t = 0; t < sel; ++t) {
    const int row = rows[size_t(t)], k = ke[row], e = el[row];
    const Rec r0{e, k, row, ev[row], kv[row], plan.AU[row], plan.l[e], plan.u[e], plan.l[k], plan.u[k], 0.0, 0.0,
                 plan.c[e]};
    const double alpha = -kv[row] / ev[row];
    const double beta = plan.AU[row] / ev[row];
    double ml = -INFINITY, mu = INFINITY;
    if (fin(plan.l[e])) { const double b = (plan.l[e] - beta) / alpha; if (alpha > 0.0) ml = b; else mu = b; }
    if (fin(plan.u[e])) { const double b = (plan.u[e] - beta) / alpha; if (alpha > 0.0) mu = b; else ml = b; }
    if (ml > mu) std::swap(ml, mu);
    const double nl = fin(ml) ? std::fmax(plan.l[k], ml) : plan.l[k];
    const double nu = fin(mu) ? std::fmin(plan.u[k], mu) : plan.u[k];
    if (nl > nu + p.bound_tol) { infeasible = true; continue; }
    if (fin(nl) && fin(nu) && nu <= nl + p.bound_tol) {
      const double at = 0.5 * (nl + nu);
      plan.l[k] = at; plan.u[k] = at;
      plan.keep_col[k] = 0;
      fixed[size_t(t)] = 1;
      fixed_obj += plan.c[k] * at;
    } else {
      plan.l[k] = nl; plan.u[k] = nu;
      plan.c[k] += plan.c[e] * alpha;
      plan.keep_row[row] = 0;
      plan.keep_col[e] = 0;
      subst[size_t(t)] = 1;
      obj += r0.ec * beta;
      Rec r = r0;
      r.nkl = nl; r.nku = nu;
      recs.push_back(r);
    }
    alpha_of[size_t(t)] = alpha;
    beta_of[size_t(t)] = beta;
    any = true;
  }
  if (infeasible) { plan.has_infeasible = true; return; }
  if (!any) return;
  if (p.record_postsolve_tape)
    for (const Rec& r : recs)
      plan.tape.add(DoubletonEquation, {r.e, r.k, r.row, 0},
                    {r.ev, r.kv, r.au, r.el, r.eu, r.kl, r.ku, r.nkl, r.nku, r.ec, 0.0, 0.0});

  // Row shifts (:1164-1189, :1191-1229), in stored column order per row: the
  // eliminated columns contribute a * beta, fixed keep columns a * value.
  std::vector<uint8_t> role(size_t(n), 0);
  std::vector<double> value(size_t(n), 0.0);
  for (int t = 0; t < sel; ++t) {
    const int row = rows[size_t(t)];
    if (subst[size_t(t)]) { role[size_t(el[row])] = 1; value[size_t(el[row])] = beta_of[size_t(t)]; }
    if (fixed[size_t(t)]) { role[size_t(ke[row])] = 1; value[size_t(ke[row])] = plan.l[ke[row]]; }
  }
  for (int i = 0; i < m; ++i) {
    if (!plan.keep_row[i]) continue;
    double shift = 0.0;
    bool touched = false;
    for (int q = A.ptr[i]; q < A.ptr[i + 1]; ++q) {
      const int j = A.idx[q];
      if (role[j] && std::fabs(A.val[q]) > zt) { shift += A.val[q] * value[j]; touched = true; }
    }
    if (touched) { plan.AL[i] -= shift; plan.AU[i] -= shift; }
  }

  // New A (:1191-1489): every row merged with the substitution deltas
  // alpha * a_(r, elim) at (r, keep), entries with |a| <= zero_tol dropped.
  if (!recs.empty()) {
    std::vector<std::vector<std::pair<int, double>>> delta(static_cast<size_t>(m));
    for (int t = 0; t < sel; ++t) {
      if (!subst[size_t(t)]) continue;
      const int row = rows[size_t(t)], e = el[row], k = ke[row];
      for (int q = ATs.ptr[e]; q < ATs.ptr[e + 1]; ++q) {
        const int r = ATs.idx[q];
        if (r != row && plan.keep_row[r] && std::fabs(ATs.val[q]) > zt)
          delta[size_t(r)].push_back({k, alpha_of[size_t(t)] * ATs.val[q]});
      }
    }
    Csr out;
    out.rows = m;
    out.cols = n;
    out.ptr.assign(size_t(m) + 1, 0);
    for (int i = 0; i < m; ++i) {
      auto& d = delta[size_t(i)];
      std::stable_sort(d.begin(), d.end(), [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
        return a.first < b.first;
      });
      int pp = A.ptr[i];
      const int pe = A.ptr[i + 1];
      size_t qq = 0;
      while (pp < pe || qq < d.size()) {
        const int sc = pp < pe ? A.idx[pp] : INT_MAX;
        const int dc = qq < d.size() ? d[qq].first : INT_MAX;
        const int col = std::min(sc, dc);
        double merged = 0.0;
        while (pp < pe && A.idx[pp] == col) merged += A.val[pp++];
        while (qq < d.size() && d[qq].first == col) merged += d[qq++].second;
        if (std::fabs(merged) > zt) { out.idx.push_back(col); out.val.push_back(merged); }
      }
      out.ptr[size_t(i) + 1] = int(out.idx.size());
    }
    plan.new_A = std::move(out);
    plan.has_new_A = true;
  }
  plan.obj_delta += obj;
  plan.obj_delta += fixed_obj;
  plan.has_row_action = !recs.empty();
  plan.has_col_action = true;
  plan.has_change = true;
}

// ---- singleton columns ------------------------------------------------------

namespace {
enum SingletonAction : uint8_t {
  kNone = 0, kSetRowSide = 1, kTightenLhs = 2, kTightenRhs = 3,
  kEliminateFree = 4, kEliminateFreeAbove = 5, kEliminateFreeBelow = 6
};

struct RowActivityCache {
  double fmin = 0.0, fmax = 0.0;
  int min_neg = 0, min_pos = 0, max_neg = 0, max_pos = 0;
  bool invalid = false;
};

// One entry's contribution (rule_singleton_columns.cu:555-654): NaN terms mark
// the row invalid and contribute nothing.
inline void cache_term(RowActivityCache& r, double a, double lj, double uj) {
  const double tmin = a >= 0.0 ? a * lj : a * uj;
  const double tmax = a >= 0.0 ? a * uj : a * lj;
  if (std::isnan(tmin) || std::isnan(tmax)) { r.invalid = true; return; }
  if (std::isinf(tmin)) (tmin < 0.0 ? r.min_neg : r.min_pos)++; else r.fmin += tmin;
  if (std::isinf(tmax)) (tmax < 0.0 ? r.max_neg : r.max_pos)++; else r.fmax += tmax;
}

// _kernel_singleton_row_activity_cache / _long_row_activity_cache
// (rule_singleton_columns.cu:555-754): rows of live length <= 1024 sum in
// stored order; longer rows give live rank k to thread k mod 256, then a
// shared-memory halving tree (stride 128 .. 1).
RowActivityCache singleton_row_cache(const Lp& lp, const Plan& plan, const Stats& s, int row) {
  RowActivityCache r;
  if (!plan.keep_row[row]) return r;
  const Csr& A = lp.A;
  if (s.row_nnz[row] <= 1024) {
    for (int p = A.ptr[row]; p < A.ptr[row + 1]; ++p) {
      const int col = A.idx[p];
      if (plan.keep_col[col]) cache_term(r, A.val[p], plan.l[col], plan.u[col]);
    }
    return r;
  }
  std::vector<RowActivityCache> part(256);
  int rank = 0;
  for (int p = A.ptr[row]; p < A.ptr[row + 1]; ++p) {
    const int col = A.idx[p];
    if (!plan.keep_col[col]) continue;
    cache_term(part[size_t(rank % 256)], A.val[p], plan.l[col], plan.u[col]);
    ++rank;
  }
  for (int stride = 128; stride > 0; stride >>= 1)
    for (int t = 0; t < stride; ++t) {
      RowActivityCache& a = part[size_t(t)];
      const RowActivityCache& b = part[size_t(t + stride)];
      a.fmin += b.fmin; a.fmax += b.fmax;
      a.min_neg += b.min_neg; a.min_pos += b.min_pos; a.max_neg += b.max_neg; a.max_pos += b.max_pos;
      a.invalid = a.invalid || b.invalid;
    }
  return part[0];
}

// _singleton_column_activity_bounds_from_cache (rule_singleton_columns.cu:756-816).
bool rest_bounds(const RowActivityCache& r, double a, double lj, double uj, double& rest_min, double& rest_max) {
  if (r.invalid) return false;
  const double tmin = a >= 0.0 ? a * lj : a * uj;
  const double tmax = a >= 0.0 ? a * uj : a * lj;
  if (std::isnan(tmin) || std::isnan(tmax)) return false;
  int min_neg = r.min_neg, min_pos = r.min_pos, max_neg = r.max_neg, max_pos = r.max_pos;
  double vmin = r.fmin, vmax = r.fmax;
  if (std::isinf(tmin)) (tmin < 0.0 ? min_neg : min_pos)--; else vmin -= tmin;
  if (std::isinf(tmax)) (tmax < 0.0 ? max_neg : max_pos)--; else vmax -= tmax;
  if (min_neg < 0 || min_pos < 0 || max_neg < 0 || max_pos < 0 || (min_neg > 0 && min_pos > 0) ||
      (max_neg > 0 && max_pos > 0))
    return false;
  rest_min = min_neg > 0 ? -INFINITY : (min_pos > 0 ? INFINITY : vmin);
  rest_max = max_neg > 0 ? -INFINITY : (max_pos > 0 ? INFINITY : vmax);
  return !std::isnan(rest_min) && !std::isnan(rest_max);
}

// _singleton_column_direct_unbounded (rule_singleton_columns.cu:516-527).
bool direct_unbounded(double cj, double a, double lhs, double rhs, double lb, double ub, double zt) {
  return (cj > zt && a > zt && !fin(lhs) && !fin(lb)) || (cj > zt && a < -zt && !fin(rhs) && !fin(lb)) ||
         (cj < -zt && a < -zt && !fin(lhs) && !fin(ub)) || (cj < -zt && a > zt && !fin(rhs) && !fin(ub));
}

// _singleton_column_implied_free_from_above / _below (rule_singleton_columns.cu:818-854).
bool free_from_above(double a, double lhs, double rhs, double ub, double rmin, double rmax, double tol) {
  if (!fin(ub)) return true;
  double implied = INFINITY;
  if (a > 0.0 && fin(rhs)) implied = (rhs - rmin) / a;
  else if (a < 0.0 && fin(lhs)) implied = (lhs - rmax) / a;
  return implied <= ub + tol;
}
bool free_from_below(double a, double lhs, double rhs, double lb, double rmin, double rmax, double tol) {
  if (!fin(lb)) return true;
  double implied = -INFINITY;
  if (a > 0.0 && fin(lhs)) implied = (lhs - rmax) / a;
  else if (a < 0.0 && fin(rhs)) implied = (rhs - rmin) / a;
  return implied >= lb - tol;
}

// _singleton_column_active_side / _ineq_action (rule_singleton_columns.cu:856-903).
uint8_t inequality_action(double cj, double a, double lhs, double rhs, bool above, bool below, double zt,
                          double& side) {
  if (above && below) {
    if ((cj > zt && a > 0.0) || (cj < -zt && a < 0.0)) side = lhs;
    else if ((cj > zt && a < 0.0) || (cj < -zt && a > 0.0)) side = rhs;
    else side = fin(lhs) ? lhs : rhs;
    return fin(side) ? kSetRowSide : kNone;
  }
  if (((cj < -zt && a > 0.0 && above) || (cj > zt && a < 0.0 && below)) && fin(rhs)) { side = rhs; return kTightenLhs; }
  if (((cj > zt && a > 0.0 && below) || (cj < -zt && a < 0.0 && above)) && fin(lhs)) { side = lhs; return kTightenRhs; }
  side = 0.0;
  return kNone;
}
}  // namespace

void rule_singleton_columns(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p) {
  // apply_rule_singleton_columns (rule_singleton_columns.cu:1562-1827).
  if (plan.has_infeasible || plan.has_unbounded || !p.enable_singleton_columns) return;
  const int m = lp.m(), n = lp.n();
  if (m == 0 || n == 0) return;
  // Precheck (_kernel_count_singleton_column_support, :1141-1155).
  bool any = false;
  for (int j = 0; j < n && !any; ++j)
    any = plan.keep_col[j] && s.singleton_col[j] && s.scol_row[j] >= 0 && plan.keep_row[size_t(s.scol_row[j])];
  if (!any) return;

  // 1. Propose (:905-1018): immutable actions, one owner per row
  //    (EliminateFree first, then the smallest column).
  std::vector<uint8_t> action(size_t(n), kNone);
  std::vector<double> side(size_t(n), 0.0);
  std::vector<int> owner(size_t(m), INT_MAX);
  std::vector<int8_t> cached(size_t(m), 0);
  std::vector<RowActivityCache> cache(static_cast<size_t>(m));
  bool unbounded = false;
  for (int j = 0; j < n; ++j) {
    if (!plan.keep_col[j] || !s.singleton_col[j]) continue;
    const int row = s.scol_row[j];
    if (row < 0 || row >= m || !plan.keep_row[row]) continue;
    const double a = s.scol_val[j];
    if (std::fabs(a) <= p.zero_tol) continue;
    int live = 0;
    for (int q = lp.A.ptr[row]; q < lp.A.ptr[row + 1] && live <= 1; ++q) live += plan.keep_col[lp.A.idx[q]] ? 1 : 0;
    if (live <= 1) continue;
    const double lhs = plan.AL[row], rhs = plan.AU[row], cj = plan.c[j];
    if (direct_unbounded(cj, a, lhs, rhs, plan.l[j], plan.u[j], p.zero_tol)) { unbounded = true; continue; }
    if (!cached[row]) { cache[row] = singleton_row_cache(lp, plan, s, row); cached[row] = 1; }
    double rmin = 0.0, rmax = 0.0;
    if (!rest_bounds(cache[row], a, plan.l[j], plan.u[j], rmin, rmax)) continue;
    const double tol = p.bound_tol;
    uint8_t act;
    double sd;
    if (fin(lhs) && fin(rhs) && std::fabs(lhs - rhs) <= tol) {
      const double x1 = (rhs - rmin) / a, x2 = (rhs - rmax) / a;
      const double ilb = std::fmin(x1, x2), iub = std::fmax(x1, x2);
      const bool above = !fin(plan.u[j]) || iub <= plan.u[j] + tol;
      const bool below = !fin(plan.l[j]) || ilb >= plan.l[j] - tol;
      if (!(above || below)) continue;
      act = above && below ? kEliminateFree : (above ? kEliminateFreeAbove : kEliminateFreeBelow);
      sd = rhs;
    } else {
      const bool above = free_from_above(a, lhs, rhs, plan.u[j], rmin, rmax, tol);
      const bool below = free_from_below(a, lhs, rhs, plan.l[j], rmin, rmax, tol);
      act = inequality_action(cj, a, lhs, rhs, above, below, p.zero_tol, sd);
      if (act == kNone) continue;
    }
    action[j] = act;
    side[j] = sd;
    const int key = act == kEliminateFree ? j - INT_MAX : j;
    owner[row] = std::min(owner[row], key);
  }
  if (unbounded) { plan.has_unbounded = true; return; }

  // 2. Stage (:1021-1073) against the unmodified plan.
  std::vector<uint8_t> row_delete(size_t(m), 0), col_delete(size_t(n), 0), lo_change(size_t(m), 0),
      hi_change(size_t(m), 0);
  std::vector<double> AL_new(plan.AL), AU_new(plan.AU), contrib(size_t(n), 0.0);
  bool any_elim = false, any_side = false;
  for (int row = 0; row < m; ++row) {
    const int j = owner[row] < 0 ? owner[row] + INT_MAX : owner[row];
    if (j < 0 || j >= n) { owner[row] = INT_MAX; continue; }
    owner[row] = j;
    const uint8_t act = action[j];
    const double lhs = plan.AL[row], rhs = plan.AU[row];
    if (act == kEliminateFree || act == kEliminateFreeAbove || act == kEliminateFreeBelow) {
      const double a = s.scol_val[j];
      contrib[j] = plan.c[j] * rhs / a;
      if (act == kEliminateFree) {
        row_delete[row] = 1;
      } else {
        const bool above = act == kEliminateFreeAbove;
        const double bound = above ? plan.l[j] : plan.u[j];
        const bool keep_lower = above ? a < 0.0 : a > 0.0;
        const double shifted = plan.AU[row] - a * bound;
        if (keep_lower) { AL_new[row] = shifted; AU_new[row] = INFINITY; }
        else { AL_new[row] = -INFINITY; AU_new[row] = shifted; }
      }
      col_delete[j] = 1;
      any_elim = true;
      continue;
    }
    if (act == kSetRowSide) {
      const double sd = side[j];
      if (!fin(lhs) || std::fabs(lhs - sd) > p.bound_tol) lo_change[row] = 1;
      if (!fin(rhs) || std::fabs(rhs - sd) > p.bound_tol) hi_change[row] = 1;
      AL_new[row] = sd;
      AU_new[row] = sd;
    } else if (act == kTightenLhs) {
      lo_change[row] = 1;
      AL_new[row] = rhs;
    } else if (act == kTightenRhs) {
      hi_change[row] = 1;
      AU_new[row] = lhs;
    }
    any_side = true;
  }
  if (!any_elim && !any_side) return;

  // Objective update of the surviving columns (:1075-1139): per column, in
  // stored (row) order of its AT entries.
  std::vector<double> c_new(plan.c);
  if (any_elim) {
    for (int col = 0; col < n; ++col) {
      if (!plan.keep_col[col] || col_delete[col]) continue;
      double updated = plan.c[col];
      for (int q = lp.AT.ptr[col]; q < lp.AT.ptr[col + 1]; ++q) {
        const int o = owner[size_t(lp.AT.idx[q])];
        if (o < 0 || o >= n || !col_delete[o]) continue;
        updated += -(plan.c[o] * lp.AT.val[q] / s.scol_val[o]);
      }
      c_new[col] = updated;
    }
  }
  // Tape before commit (:1191-1560, :459-508).
  if (any_elim && p.record_postsolve_tape) {
    for (int row = 0; row < m; ++row) {
      const int col = owner[row];
      if (col < 0 || col >= n || !col_delete[col]) continue;
      double pivot = 0.0;
      std::vector<int> sidx;
      std::vector<double> sval;
      for (int q = lp.A.ptr[row]; q < lp.A.ptr[row + 1]; ++q) {
        const int rc = lp.A.idx[q];
        if (rc == col) pivot = lp.A.val[q];
        else if (plan.keep_col[rc]) { sidx.push_back(rc); sval.push_back(lp.A.val[q]); }
      }
      if (std::fabs(pivot) <= p.zero_tol) continue;
      std::vector<int> idx{col, row, int(sidx.size())};
      idx.insert(idx.end(), sidx.begin(), sidx.end());
      std::vector<double> val{pivot, side[col], plan.l[col], plan.u[col], plan.c[col], row_delete[row] ? 1.0 : 0.0};
      val.insert(val.end(), sval.begin(), sval.end());
      plan.tape.add(SingletonColumnSubstitution, idx, val);
    }
  }
  if (any_side && p.record_postsolve_tape)
    for (int row = 0; row < m; ++row)
      if (lo_change[row] || hi_change[row]) plan.tape.add(RowDualShift, {row}, {0.0});
  // Commit (:1157-1189).
  for (int row = 0; row < m; ++row) {
    if (row_delete[row]) plan.keep_row[row] = 0;
    if (owner[row] >= 0 && owner[row] < n) { plan.AL[row] = AL_new[row]; plan.AU[row] = AU_new[row]; }
  }
  for (int j = 0; j < n; ++j) {
    if (col_delete[j]) plan.keep_col[j] = 0;
    if (any_elim && plan.keep_col[j]) plan.c[j] = c_new[j];
  }
  plan.obj_delta += domain_objective(contrib, plan);
  plan.has_row_action = true;
  plan.has_col_action = plan.has_col_action || any_elim;
  plan.has_change = true;
}

namespace {
inline void term_interval(double a, double lj, double uj, double& tmin, double& tmax) {
  if (a >= 0.0) { tmin = a * lj; tmax = a * uj; } else { tmin = a * uj; tmax = a * lj; }
}
inline double residual_min(double fin_sum, int ninf, double t) {
  if (fin(t)) return ninf == 0 ? fin_sum - t : -INFINITY;
  if (t < 0.0) return ninf > 1 ? -INFINITY : fin_sum;
  return fin_sum;
}
inline double residual_max(double fin_sum, int pinf, double t) {
  if (fin(t)) return pinf == 0 ? fin_sum - t : INFINITY;
  if (t > 0.0) return pinf > 1 ? INFINITY : fin_sum;
  return fin_sum;
}
// Implied bounds of column j from row i (rule_bound_strengthening.cu:349-430).
inline void implied_bounds(double a, double lj, double uj, double al, double au, double mn, double mx,
                           int ni, int pi, double& il, double& iu) {
  double tmin, tmax;
  term_interval(a, lj, uj, tmin, tmax);
  const double rmin = residual_min(mn, ni, tmin);
  const double rmax = residual_max(mx, pi, tmax);
  il = -INFINITY;
  iu = INFINITY;
  if (a > 0.0) {
    if (fin(al) && fin(rmax)) il = (al - rmax) / a;
    if (fin(au) && fin(rmin)) iu = (au - rmin) / a;
  } else {
    if (fin(au) && fin(rmin)) il = (au - rmin) / a;
    if (fin(al) && fin(rmax)) iu = (al - rmax) / a;
  }
}
}  // namespace

void rule_bound_strengthening(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p) {
  // apply_rule_bound_strengthening (rule_bound_strengthening.cu:1176-1557):
  // one Jacobi round of activity-based implied bounds.
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (m == 0 || n == 0) return;
  std::vector<double> cl(plan.l), cu(plan.u);
  std::vector<double> mn(m), mx(m);
  std::vector<int> ni(m), pi(m);
  row_activity_summary(lp.A, plan.l, plan.u, p.zero_tol, plan.keep_row.data(), plan.keep_col.data(),
                       s.row_nnz.data(), mn.data(), mx.data(), ni.data(), pi.data());
  for (int i = 0; i < m; ++i) {
    if (!plan.keep_row[i] || s.row_nnz[i] <= 1) continue;
    for (int q = lp.A.ptr[i]; q < lp.A.ptr[i + 1]; ++q) {
      const int j = lp.A.idx[q];
      if (!plan.keep_col[j]) continue;
      const double a = lp.A.val[q];
      if (std::fabs(a) <= p.zero_tol) continue;
      const double ol = plan.l[j], ou = plan.u[j];
      double il, iu;
      implied_bounds(a, ol, ou, plan.AL[i], plan.AU[i], mn[i], mx[i], ni[i], pi[i], il, iu);
      double nl = ol, nu = ou;
      if (fin(il)) nl = std::fmax(nl, il);
      if (fin(iu)) nu = std::fmin(nu, iu);
      if (nl > ol) max_into(cl[j], nl);
      if (nu < ou) min_into(cu[j], nu);
    }
  }
  std::vector<double> cmax(n);
  col_max_abs(lp.AT, plan.keep_row.data(), cmax.data());
  const std::vector<double>& refl = plan.ref_l ? *plan.ref_l : plan.l;
  const std::vector<double>& refu = plan.ref_u ? *plan.ref_u : plan.u;
  const double ft = p.feasibility_tol;
  std::vector<double> fl(n), fu(n), fixv(n, 0.0);
  std::vector<uint8_t> lch(n, 0), uch(n, 0), fx(n, 0);
  bool f_infeasible = false, f_changed = false, f_fixed = false;
  // _kernel_finalize_bound_strengthening (rule_bound_strengthening.cu:646-796).
  for (int j = 0; j < n; ++j) {
    const double lj = plan.l[j], uj = plan.u[j];
    if (!plan.keep_col[j]) { fl[j] = lj; fu[j] = uj; continue; }
    double cand_l = cl[j], cand_u = cu[j];
    const double vmax = cmax[j];
    double nl = lj, nu = uj;
    uint8_t lc = 0, uc = 0, fj = 0;
    double fat = 0.0;
    double el = lj, eu = uj;
    if (fin(cand_l)) el = std::fmax(el, cand_l);
    if (fin(cand_u)) eu = std::fmin(eu, cand_u);
    if (el > eu + ft) { f_infeasible = true; continue; }
    const bool was_free = !fin(refl[j]) && !fin(refu[j]);
    const bool box = fin(cand_l) && fin(cand_u);
    const bool zero_cost = std::fabs(plan.c[j]) <= p.zero_tol;
    const bool nearly_fixed = box && (cand_u <= cand_l || (cand_u - cand_l) * vmax <= ft);
    if (p.bound_strengthening_preserve_free_zero_cost && was_free && box && zero_cost && !nearly_fixed) {
      cand_l = lj;
      cand_u = uj;
    }
    if (fin(cand_l) && cand_l > lj && fin(uj)) {
      if (cand_l >= uj + ft) { f_infeasible = true; continue; }
      if (cand_l >= uj || (uj - cand_l) * vmax <= ft) { fj = 1; fat = uj; nl = uj; nu = uj; }
    }
    if (!fj && fin(cand_l) && cand_l > lj) {
      const bool tighten = !fin(lj) || ((cand_l - lj > ft * 1.0e4) && (cand_l - lj > 1.0e-2 * std::fabs(lj)));
      if (tighten) {
        if (cand_l != std::nearbyint(cand_l)) cand_l -= 0.5 * ft * std::fabs(cand_l);
        nl = cand_l;
        lc = 1;
      }
    }
    if (!fj && fin(cand_u) && cand_u < uj && fin(nl)) {
      if (cand_u <= nl - ft) { f_infeasible = true; continue; }
      if (cand_u <= nl || (cand_u - nl) * vmax <= ft) { fj = 1; fat = nl; nu = nl; }
    }
    if (!fj && fin(cand_u) && cand_u < uj) {
      const bool tighten = !fin(uj) || ((uj - cand_u > ft * 1.0e4) && (uj - cand_u > 1.0e-2 * std::fabs(uj)));
      if (tighten) {
        if (cand_u != std::nearbyint(cand_u))
          cand_u += p.bound_strengthening_upper_relaxation_factor * ft * std::fabs(cand_u);
        nu = cand_u;
        uc = 1;
      }
    }
    if (fj) { lc = uc = 0; f_fixed = true; }
    if (lc || uc) f_changed = true;
    fl[j] = nl; fu[j] = nu; lch[j] = lc; uch[j] = uc; fx[j] = fj; fixv[j] = fat;
  }
  if (f_infeasible) { plan.has_infeasible = true; return; }
  if (!f_changed && !f_fixed) return;
  if (p.record_postsolve_tape && f_changed) {
    // Support rows (rule_bound_strengthening.cu:815-960): the smallest live row
    // whose implied bound reproduces the finalized bound within support_tol.
    const double support_tol = std::fmax(10.0 * p.bound_tol, 1.0e-10);
    Tape seg;
    for (int j = 0; j < n; ++j) {
      if (!lch[j] && !uch[j]) continue;
      int sl = INT_MAX, su = INT_MAX;
      for (int q = lp.AT.ptr[j]; q < lp.AT.ptr[j + 1]; ++q) {
        const int i = lp.AT.idx[q];
        if (!plan.keep_row[i] || s.row_nnz[i] <= 1) continue;
        const double a = lp.AT.val[q];
        if (std::fabs(a) <= p.zero_tol) continue;
        double il, iu;
        implied_bounds(a, plan.l[j], plan.u[j], plan.AL[i], plan.AU[i], mn[i], mx[i], ni[i], pi[i], il, iu);
        if (lch[j] && fl[j] > plan.l[j] + p.bound_tol && fin(il) && std::fabs(il - fl[j]) <= support_tol)
          sl = std::min(sl, i);
        if (uch[j] && fu[j] < plan.u[j] - p.bound_tol && fin(iu) && std::fabs(iu - fu[j]) <= support_tol)
          su = std::min(su, i);
      }
      double cur_l = plan.l[j];
      const double cur_u = plan.u[j];
      if (lch[j]) {
        if (sl != INT_MAX) seg.add(RowImpliedBoundChange, {j, sl}, {cur_l, cur_u, fl[j], cur_u});
        else seg.add(VariableBoundChange, {j}, {cur_l, cur_u, fl[j], cur_u});
        cur_l = fl[j];
      }
      if (uch[j]) {
        if (su != INT_MAX) seg.add(RowImpliedBoundChange, {j, su}, {cur_l, cur_u, cur_l, fu[j]});
        else seg.add(VariableBoundChange, {j}, {cur_l, cur_u, cur_l, fu[j]});
      }
    }
    plan.tape.append(seg);
  }
  for (int j = 0; j < n; ++j) {
    plan.l[j] = fl[j];
    plan.u[j] = fu[j];
    if (fx[j]) plan.keep_col[j] = 0;
  }
  bool empty_infeasible = false;
  if (f_fixed) {
    const std::vector<double> shift = row_shift_gather(lp, plan.keep_row, fx, fixv, false);
    for (int i = 0; i < m; ++i) { plan.AL[i] -= shift[i]; plan.AU[i] -= shift[i]; }
    for (int i = 0; i < m; ++i) {
      if (!plan.keep_row[i]) continue;
      int cnt = 0;
      for (int q = lp.A.ptr[i]; q < lp.A.ptr[i + 1]; ++q) cnt += plan.keep_col[lp.A.idx[q]] != 0;
      if (cnt != 0) continue;
      if (plan.AL[i] <= ft && plan.AU[i] >= -ft) plan.keep_row[i] = 0; else empty_infeasible = true;
    }
  }
  if (empty_infeasible) { plan.has_infeasible = true; return; }
  double obj_delta = 0.0;
  if (f_fixed) {
    // append_compact_fixed_variable_tape_from_device (fixed_variable_tape.cu:141-327).
    long double acc = 0.0L;
    Tape seg;
    for (int j = 0; j < n; ++j) {
      if (!fx[j]) continue;
      acc += (long double)plan.c[j] * (long double)fixv[j];
      if (!p.record_postsolve_tape) continue;
      std::vector<int> ii{j};
      std::vector<double> vv{fixv[j], plan.c[j]};
      for (int q = lp.AT.ptr[j]; q < lp.AT.ptr[j + 1]; ++q)
        if (plan.keep_row[lp.AT.idx[q]]) { ii.push_back(lp.AT.idx[q]); vv.push_back(lp.AT.val[q]); }
      seg.add(FixedVariable, ii, vv);
    }
    plan.tape.append(seg);
    obj_delta = double(acc);
  }
  plan.obj_delta += obj_delta;
  plan.has_row_action = plan.has_row_action || f_fixed;
  plan.has_col_action = plan.has_col_action || f_fixed;
  plan.has_change = true;
}

void rule_redundant_rows(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p) {
  // apply_rule_infeasible_and_redundant_rows (rule_infeasible_and_redundant_rows.cu:178-331).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m();
  if (m == 0) return;
  std::vector<double> mn(static_cast<size_t>(m)), mx(static_cast<size_t>(m));
  row_plain_minmax(lp.A, plan.l, plan.u, plan.keep_row.data(), plan.keep_col.data(), s.row_nnz.data(), mn.data(),
                   mx.data());
  const double tol = p.bound_tol;
  std::vector<uint8_t> full(size_t(m), 0), dl(size_t(m), 0), du(size_t(m), 0);
  bool infeasible = false, any = false, any_full = false;
  for (int i = 0; i < m; ++i) {
    if (!plan.keep_row[i] || s.row_nnz[i] <= 1) continue;
    const double al = plan.AL[i], au = plan.AU[i];
    const bool lf = fin(al), uf = fin(au);
    if (lf && uf && std::fabs(au - al) <= tol) continue;
    const double lo = mn[i], hi = mx[i];
    if ((lf && hi < al - tol) || (uf && lo > au + tol)) { infeasible = true; continue; }
    const bool li = !lf || lo >= al - tol, ui = !uf || hi <= au + tol;
    if (li && ui) { full[i] = 1; any = any_full = true; }
    else if (lf && li) { dl[i] = 1; any = true; }
    else if (uf && ui) { du[i] = 1; any = true; }
  }
  if (infeasible) { plan.has_infeasible = true; return; }
  if (!any) return;
  for (int i = 0; i < m; ++i) {
    if (full[i]) plan.keep_row[i] = 0;
    if (dl[i]) plan.AL[i] = -INFINITY;
    if (du[i]) plan.AU[i] = INFINITY;
  }
  plan.has_row_action = true;
  plan.has_redundant_row_deletion = plan.has_redundant_row_deletion || any_full;
  plan.has_row_deletion = plan.has_row_deletion || any_full;
  plan.has_change = true;
}

void rule_dual_fix(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p) {
  // apply_rule_dual_fix (rule_dual_fix.cu:203-645) on the deferred plan.
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int n = lp.n(), m = lp.m();
  if (n == 0) return;
  std::vector<uint8_t> fixed(size_t(n), 0), inf(size_t(n), 0);
  std::vector<double> fval(size_t(n), 0.0), contrib(size_t(n), 0.0);
  int status0 = 0;
  bool any = false, any_inf = false;
  const double zt = p.zero_tol;
  for (int j = 0; j < n; ++j) {
    if (!plan.keep_col[j]) continue;
    const double lj = plan.l[j], uj = plan.u[j];
    if (lj > uj + p.bound_tol) { status0 = std::max(status0, 1); continue; }
    const double cj = plan.c[j];
    if (std::fabs(cj) > zt && s.col_nnz[j] > p.dual_fix_max_nonzero_cost_col_degree) continue;
    bool down = false, up = false;
    for (int q = lp.AT.ptr[j]; q < lp.AT.ptr[j + 1]; ++q) {
      const int row = lp.AT.idx[q];
      if (!plan.keep_row[row]) continue;
      const double a = lp.AT.val[q];
      if (a > zt) { down = down || fin(plan.AL[row]); up = up || fin(plan.AU[row]); }
      else if (a < -zt) { down = down || fin(plan.AU[row]); up = up || fin(plan.AL[row]); }
      if (down && up) break;
    }
    bool f = false, fi = false;
    double v = 0.0;
    if (cj > zt) {
      if (!down) { if (fin(lj)) { v = lj; f = true; } else { status0 = std::max(status0, 2); continue; } }
    } else if (cj < -zt) {
      if (!up) { if (fin(uj)) { v = uj; f = true; } else { status0 = std::max(status0, 2); continue; } }
    } else if (std::fabs(cj) <= zt) {
      if (!down) { f = true; if (fin(lj)) v = lj; else { v = -INFINITY; fi = true; } }
      else if (!up) { f = true; if (fin(uj)) v = uj; else { v = INFINITY; fi = true; } }
    }
    if (f) {
      fixed[j] = 1; inf[j] = fi; fval[j] = v; contrib[j] = fi ? 0.0 : cj * v;
      any = true;
      any_inf = any_inf || fi;
    }
  }
  if (status0 == 1) { plan.has_infeasible = true; return; }
  if (status0 == 2) { plan.has_unbounded = true; return; }
  if (!any) return;
  std::vector<uint8_t> finite_fixed(size_t(n), 0);
  for (int j = 0; j < n; ++j) finite_fixed[size_t(j)] = fixed[size_t(j)] && !inf[size_t(j)];
  const std::vector<double> shift = row_shift_gather(lp, plan.keep_row, finite_fixed, fval, false);
  std::vector<uint8_t> remove(size_t(m), 0);
  bool row_changed = false;
  for (int j = 0; j < n; ++j) {
    if (!(fixed[j] && inf[j])) continue;
    for (int q = lp.AT.ptr[j]; q < lp.AT.ptr[j + 1]; ++q)
      if (plan.keep_row[lp.AT.idx[q]]) { remove[size_t(lp.AT.idx[q])] = 1; row_changed = true; }
  }
  if (p.record_postsolve_tape && any_inf) {
    // infinite_counts / infinite_pack (device_recovery.cu:350-412): rows of the
    // column with their entries restricted to the rule-entry column domain.
    const std::vector<uint8_t>& entry = *plan.rule_entry_keep_col;
    Tape seg;
    for (int j = 0; j < n; ++j) {
      if (!(fixed[j] && inf[j])) continue;
      const bool pos = fval[j] > 0;
      std::vector<int> ii{pos ? 1 : -1, j, 0};
      std::vector<double> vv{pos ? plan.l[j] : plan.u[j]};
      int active = 0;
      for (int q = lp.AT.ptr[j]; q < lp.AT.ptr[j + 1]; ++q) {
        const int row = lp.AT.idx[q];
        if (!plan.keep_row[row]) continue;
        ++active;
        const size_t header = ii.size();
        ii.push_back(0);
        vv.push_back(fin(plan.AL[row]) ? plan.AL[row] : plan.AU[row]);
        for (int t = lp.A.ptr[row]; t < lp.A.ptr[row + 1]; ++t) {
          if (!entry[size_t(lp.A.idx[t])]) continue;
          ++ii[header];
          ii.push_back(lp.A.idx[t]);
          vv.push_back(lp.A.val[t]);
        }
      }
      ii[2] = active;
      seg.add(InfiniteBoundDualFix, ii, vv);
    }
    plan.tape.append(seg);
  }
  for (int j = 0; j < n; ++j)
    if (fixed[j]) { plan.l[j] = fval[j]; plan.u[j] = fval[j]; plan.keep_col[j] = 0; }
  for (int i = 0; i < m; ++i) {
    plan.AL[i] -= shift[i];
    plan.AU[i] -= shift[i];
    if (remove[i]) plan.keep_row[i] = 0;
  }
  plan.obj_delta += domain_objective(contrib, plan);
  plan.has_row_action = plan.has_row_action || row_changed;
  plan.has_col_action = true;
  plan.has_change = true;
}

namespace {
// (hash, index) pairs of live rows / columns sorted ascending.
std::vector<std::pair<uint64_t, int>> sorted_groups(std::vector<uint64_t> h, const std::vector<uint8_t>& keep) {
  std::vector<std::pair<uint64_t, int>> v;
  for (size_t i = 0; i < keep.size(); ++i)
    if (keep[i]) v.push_back({h[i], int(i)});
  std::sort(v.begin(), v.end());
  return v;
}

// _parallel_row_ratio (rule_parallel_rows.cu:346-377).
bool row_ratio(const Csr& A, int i, int k, double tol, const std::vector<uint8_t>& keep_col, double* out) {
  std::vector<int> L, R;
  for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) if (keep_col[A.idx[p]]) L.push_back(p);
  for (int p = A.ptr[k]; p < A.ptr[k + 1]; ++p) if (keep_col[A.idx[p]]) R.push_back(p);
  if (L.empty() && R.empty()) { *out = 1.0; return true; }
  double ratio = 0.0;
  bool set = false;
  size_t a = 0;
  for (; a < L.size() && a < R.size(); ++a) {
    if (A.idx[L[a]] != A.idx[R[a]]) return false;
    const double ai = A.val[L[a]], ak = A.val[R[a]];
    if (!set) {
      if (std::fabs(ak) <= tol) return false;
      ratio = ai / ak;
      set = true;
    }
    if (std::fabs(ai - ratio * ak) > tol) return false;
  }
  *out = ratio;
  return set && a == L.size() && a == R.size();
}

// _parallel_column_ratio (rule_parallel_columns.cu:262-321).
bool col_ratio(const Csr& AT, int j, int k, const std::vector<uint8_t>& keep_row, double zt, double ct, double* out) {
  auto live = [&](int c) {
    std::vector<int> v;
    for (int p = AT.ptr[c]; p < AT.ptr[c + 1]; ++p)
      if (keep_row[AT.idx[p]] && std::fabs(AT.val[p]) > zt) v.push_back(p);
    return v;
  };
  const auto J = live(j), K = live(k);
  double ratio = 0.0;
  bool set = false;
  size_t a = 0;
  for (; a < J.size() && a < K.size(); ++a) {
    if (AT.idx[J[a]] != AT.idx[K[a]]) return false;
    const double aj = AT.val[J[a]], ak = AT.val[K[a]];
    if (!set) {
      if (std::fabs(aj) <= zt) return false;
      ratio = ak / aj;
      if (std::fabs(ratio) <= zt || !fin(ratio)) return false;
      set = true;
    }
    const double expected = ratio * aj;
    const double scale = std::fmax(std::fabs(ak), std::fabs(expected));
    if (!fin(expected) || std::fabs(ak - expected) > ct * scale) return false;
  }
  if (a < J.size() || a < K.size() || !set) return false;
  *out = ratio;
  return true;
}

void scaled(double lo, double hi, double r, double& sl, double& su) {
  const double a = lo * r, b = hi * r;
  if (r >= 0.0) { sl = a; su = b; } else { sl = b; su = a; }
}
}  // namespace

void rule_parallel_rows(Plan& plan, const Lp& lp, const Stats&, const gpp_params& p) {
  // apply_rule_parallel_rows (rule_parallel_rows.cu:643-888).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m();
  if (m <= 1) return;
  const int mode = int64_t(lp.A.nnz()) > 32LL * m ? 1 : 0;
  std::vector<uint64_t> h(static_cast<size_t>(m));
  for (int i = 0; i < m; ++i)
    h[size_t(i)] = plan.keep_row[i] ? row_hash_tol(lp.A, i, plan.keep_col.data(), mode, p.zero_tol) : uint64_t(i);
  const auto g = sorted_groups(h, plan.keep_row);
  const double ct = p.zero_tol, it = p.feasibility_tol;
  struct Rec { int step, kept, del; double v[5]; };
  std::vector<Rec> recs;
  std::vector<uint8_t> del(size_t(m), 0);
  for (size_t s = 0; s < g.size();) {
    size_t e = s;
    while (e + 1 < g.size() && g[e + 1].first == g[s].first) ++e;
    const size_t s0 = s;
    s = e + 1;
    if (e == s0) continue;
    int seed = -1;
    bool seed_eq = false;
    for (size_t a = s0; a <= e; ++a) {
      const int row = g[a].second;
      if (!plan.keep_row[row]) continue;
      const bool eq = fin(plan.AL[row]) && fin(plan.AU[row]) && std::fabs(plan.AL[row] - plan.AU[row]) <= it;
      if (seed < 0 || (eq && !seed_eq)) { seed = row; seed_eq = eq; }
    }
    if (seed < 0) continue;
    int rep = seed;
    double rsl = plan.AL[seed], rsu = plan.AU[seed];
    for (size_t a = s0; a <= e; ++a) {
      const int row = g[a].second;
      if (row == seed || !plan.keep_row[row]) continue;
      double r;
      if (!row_ratio(lp.A, seed, row, ct, plan.keep_col, &r)) continue;
      double sl, su;
      scaled(plan.AL[row], plan.AU[row], r, sl, su);
      if (rsl <= sl + it && su <= rsu + it) { rep = row; rsl = sl; rsu = su; }
    }
    double rl = plan.AL[rep], ru = plan.AU[rep];
    bool found = false;
    int step = 0;
    for (size_t a = s0; a <= e; ++a) {
      const int row = g[a].second;
      if (row == rep || !plan.keep_row[row]) continue;
      double r;
      if (!row_ratio(lp.A, rep, row, ct, plan.keep_col, &r)) continue;
      found = true;
      double sl, su;
      scaled(plan.AL[row], plan.AU[row], r, sl, su);
      if (std::fmax(rl, sl) > std::fmin(ru, su) + it) { plan.has_infeasible = true; return; }
      ++step;
      recs.push_back({step, rep, row, {r, rl, ru, plan.AL[row], plan.AU[row]}});
      rl = std::fmax(rl, sl);
      ru = std::fmin(ru, su);
      del[size_t(row)] = 1;
    }
    if (found) { plan.AL[rep] = rl; plan.AU[rep] = ru; }
  }
  if (recs.empty()) return;
  for (int i = 0; i < m; ++i) if (del[size_t(i)]) plan.keep_row[i] = 0;
  if (p.record_postsolve_tape) {
    std::sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) {
      return a.step != b.step ? a.step < b.step : a.del < b.del;
    });
    Tape seg;
    for (const auto& r : recs)
      seg.add(ParallelRow, {r.kept, r.del}, {r.v[0], r.v[1], r.v[2], r.v[3], r.v[4]});
    plan.tape.append(seg);
  }
  plan.has_row_action = plan.has_change = true;
}

void rule_parallel_columns(Plan& plan, const Lp& lp, const Stats&, const gpp_params& p) {
  // apply_rule_parallel_columns (rule_parallel_columns.cu:725-1127).
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (n <= 1) return;
  std::vector<uint64_t> h(static_cast<size_t>(n));
  for (int j = 0; j < n; ++j)
    h[size_t(j)] = plan.keep_col[j] ? col_hash(lp.AT, j, plan.keep_row.data(), p.zero_tol) : uint64_t(j);
  const auto g = sorted_groups(h, plan.keep_col);
  const double zt = p.zero_tol, ct = std::fmax(p.zero_tol, p.bound_tol), ot = ct;
  const double max_abs = p.parallel_columns_max_abs_ratio;
  const bool guard = fin(max_abs) && p.parallel_columns_scale_guard_min_groups > 1;
  auto guarded = [](double r, double mx) {
    const double a = std::fabs(r);
    return fin(mx) && (mx < 1.0 || a > mx || a * mx < 1.0);
  };
  int guard_count = 0;
  if (guard) {
    for (size_t s = 0; s < g.size();) {
      size_t e = s;
      while (e + 1 < g.size() && g[e + 1].first == g[s].first) ++e;
      const size_t s0 = s;
      s = e + 1;
      const int size = int(e - s0 + 1);
      if (size < 2 || size > p.parallel_columns_scale_guard_max_group_size) continue;
      bool hit = false;
      for (size_t a = s0; a < e && !hit; ++a) {
        const int j = g[a].second;
        for (size_t b = a + 1; b <= e; ++b) {
          const int k = g[b].second;
          double r;
          if (!col_ratio(lp.AT, j, k, plan.keep_row, zt, ct, &r)) continue;
          if (std::fabs(plan.c[k] - r * plan.c[j]) > ot) continue;
          if (max_abs < 1.0 || std::fabs(r) > max_abs || std::fabs(r) * max_abs < 1.0) { hit = true; break; }
        }
      }
      if (hit) ++guard_count;
    }
  }
  const double active_max = guard && guard_count < p.parallel_columns_scale_guard_min_groups ? INFINITY : max_abs;
  std::vector<uint8_t> del(size_t(n), 0), fixed(size_t(n), 0);
  std::vector<double> fval(size_t(n), 0.0);
  struct Rec { int del, kept; double v[5]; };
  std::vector<Rec> recs;
  bool any_fixed = false;
  for (size_t s = 0; s < g.size();) {
    size_t e = s;
    while (e + 1 < g.size() && g[e + 1].first == g[s].first) ++e;
    const size_t s0 = s;
    s = e + 1;
    if (e == s0) continue;
    for (size_t a = s0; a < e; ++a) {
      const int j = g[a].second;
      if (!plan.keep_col[j] || del[size_t(j)] || fixed[size_t(j)]) continue;
      for (size_t b = a + 1; b <= e; ++b) {
        const int k = g[b].second;
        if (!plan.keep_col[k] || del[size_t(k)] || fixed[size_t(k)]) continue;
        double r;
        if (!col_ratio(lp.AT, j, k, plan.keep_row, zt, ct, &r)) continue;
        if (guarded(r, active_max)) continue;
        const double gap = plan.c[k] - r * plan.c[j];
        const double tl = plan.l[j], tu = plan.u[j], sl = plan.l[k], su = plan.u[k];
        if (std::fabs(gap) <= ot) {
          recs.push_back({k, j, {r, sl, su, tl, tu}});
          double nl = -INFINITY, nu = INFINITY;
          if (r > 0.0) { if (fin(tl) && fin(sl)) nl = tl + r * sl; }
          else if (fin(tl) && fin(su)) nl = tl + r * su;
          if (r > 0.0) { if (fin(tu) && fin(su)) nu = tu + r * su; }
          else if (fin(tu) && fin(sl)) nu = tu + r * sl;
          plan.l[j] = nl;
          plan.u[j] = nu;
          del[size_t(k)] = 1;
          continue;
        }
        bool k_lo = false, k_hi = false, j_lo = false, j_hi = false;
        if (gap > ot) {
          if (r > 0.0) { k_lo = !fin(tu); j_hi = !fin(sl); } else { k_lo = !fin(tl); j_lo = !fin(sl); }
        } else {
          if (r > 0.0) { k_hi = !fin(tl); j_lo = !fin(su); } else { k_hi = !fin(tu); j_hi = !fin(su); }
        }
        if (k_lo) {
          if (!fin(sl)) { plan.has_unbounded = true; return; }
          fixed[size_t(k)] = 1; fval[size_t(k)] = sl; any_fixed = true;
          continue;
        } else if (k_hi) {
          if (!fin(su)) { plan.has_unbounded = true; return; }
          fixed[size_t(k)] = 1; fval[size_t(k)] = su; any_fixed = true;
          continue;
        }
        if (j_lo) {
          if (!fin(tl)) { plan.has_unbounded = true; return; }
          fixed[size_t(j)] = 1; fval[size_t(j)] = tl; any_fixed = true;
          break;
        } else if (j_hi) {
          if (!fin(tu)) { plan.has_unbounded = true; return; }
          fixed[size_t(j)] = 1; fval[size_t(j)] = tu; any_fixed = true;
          break;
        }
      }
    }
  }
  if (recs.empty() && !any_fixed) return;
  if (!recs.empty() && p.record_postsolve_tape) {
    std::sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) { return a.del < b.del; });
    Tape seg;
    for (const auto& r : recs) seg.add(ParallelColumn, {r.del, r.kept}, {r.v[0], r.v[1], r.v[2], r.v[3], r.v[4]});
    plan.tape.append(seg);
  }
  std::vector<double> shift(size_t(m), 0.0);
  if (any_fixed) {
    if (p.record_postsolve_tape) {
      Tape seg;
      for (int j = 0; j < n; ++j) {
        if (!fixed[size_t(j)]) continue;
        std::vector<int> ii{j};
        std::vector<double> vv{fval[size_t(j)], plan.c[j]};
        for (int q = lp.AT.ptr[j]; q < lp.AT.ptr[j + 1]; ++q)
          if (plan.keep_row[lp.AT.idx[q]]) { ii.push_back(lp.AT.idx[q]); vv.push_back(lp.AT.val[q]); }
        seg.add(FixedVariable, ii, vv);
      }
      plan.tape.append(seg);
    }
    shift = row_shift_gather(lp, plan.keep_row, fixed, fval, false);
    plan.has_row_action = true;
  }
  std::vector<double> contrib(size_t(n), 0.0);
  for (int q = 0; q < n; ++q) {
    if (!(del[size_t(q)] || fixed[size_t(q)])) continue;
    plan.keep_col[q] = 0;
    if (fixed[size_t(q)]) {
      plan.l[q] = fval[size_t(q)];
      plan.u[q] = fval[size_t(q)];
      contrib[size_t(q)] = plan.c[q] * fval[size_t(q)];
    }
  }
  if (any_fixed)
    for (int i = 0; i < m; ++i) { plan.AL[i] -= shift[size_t(i)]; plan.AU[i] -= shift[size_t(i)]; }
  plan.obj_delta += any_fixed ? det_sum(contrib) : 0.0;
  plan.has_col_action = plan.has_change = true;
}

void rule_column_domination(Plan& plan, const Lp& lp, const gpp_params& p) {
  // analyze_column_domination / build_column_domination_plan
  // (rule_column_domination.cu:248-379): strict unit set covering only.
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  const int nnz = lp.A.ptr[size_t(m)];
  const int min_fixed = std::max(1, p.column_domination_min_fixed_cols);
  if (m <= 0 || nnz <= 0 || n < min_fixed) return;
  for (int i = 0; i < m; ++i) {
    if (plan.AL[size_t(i)] != 1.0 || !(std::isinf(plan.AU[size_t(i)]) && plan.AU[size_t(i)] > 0.0)) return;
    bool witness = false;
    for (int q = lp.A.ptr[size_t(i)]; q < lp.A.ptr[size_t(i) + 1] && !witness; ++q)
      witness = plan.c[size_t(lp.A.idx[size_t(q)])] == 1.0;
    if (!witness) return;
  }
  for (int j = 0; j < n; ++j) {
    const double cj = plan.c[size_t(j)];
    if (plan.l[size_t(j)] != 0.0 || plan.u[size_t(j)] != 1.0) return;
    if (!(std::isfinite(cj) && cj >= 1.0 && std::floor(cj) == cj)) return;
  }
  for (int q = 0; q < nnz; ++q)
    if (lp.A.val[size_t(q)] != 1.0 || lp.AT.val[size_t(q)] != 1.0) return;
  std::vector<uint8_t> dominated(size_t(n), 0);
  int count = 0;
  for (int j = 0; j < n; ++j) {
    dominated[size_t(j)] = plan.c[size_t(j)] > double(lp.AT.ptr[size_t(j) + 1] - lp.AT.ptr[size_t(j)]);
    count += dominated[size_t(j)];
  }
  if (count < min_fixed || double(count) / double(n) + 1.0e-15 < p.column_domination_min_candidate_ratio) return;
  for (int j = 0; j < n; ++j)
    if (dominated[size_t(j)]) {
      plan.keep_col[size_t(j)] = 0;
      plan.l[size_t(j)] = 0.0;
      plan.u[size_t(j)] = 0.0;
    }
  plan.has_col_action = plan.has_change = true;
}


// ---- projected auxiliaries ------------------------------------------------
// Two-row variable elimination (rule_two_row_variable_elimination.cu) and
// zero-cost product variables (rule_zero_cost_product_variables.cu): the
// detectors see the plan's masks (the deletions of earlier rules of the
// Startup batch), selected columns leave with their rows, and each leaves a
// projected-column record (the device layout of device_recovery.cu:433-476).
namespace {

constexpr int kMaxCertified = 8;

struct Expr {
  double constant = 0.0;
  std::vector<int> cols;
  std::vector<double> coeffs;
};

bool add_term(Expr& e, int col, double coeff, size_t capacity) {
  if (!std::isfinite(coeff)) return false;
  for (size_t k = 0; k < e.cols.size(); ++k)
    if (e.cols[k] == col) { e.coeffs[k] += coeff; return std::isfinite(e.coeffs[k]); }
  if (e.cols.size() >= capacity) return false;
  e.cols.push_back(col);
  e.coeffs.push_back(coeff);
  return true;
}

bool margin_le(double lhs, double rhs, double tol) {
  if (!std::isfinite(lhs) || !std::isfinite(rhs)) return false;
  return rhs - lhs >= tol * (1.0 + std::fmax(std::fabs(lhs), std::fabs(rhs)));
}

// The K rows of column j that the plan keeps, or empty.
std::vector<int> kept_rows(const Lp& lp, const Plan& plan, int j, size_t K) {
  std::vector<int> out;
  for (int q = lp.AT.ptr[size_t(j)]; q < lp.AT.ptr[size_t(j) + 1]; ++q) {
    const int i = lp.AT.idx[size_t(q)];
    if (!plan.keep_row[size_t(i)]) continue;
    if (out.size() == K) return {};
    out.push_back(i);
  }
  return out.size() == K ? out : std::vector<int>{};
}

int live_in_row(const Lp& lp, const Plan& plan, int i, int cap) {
  int live = 0;
  for (int q = lp.A.ptr[size_t(i)]; q < lp.A.ptr[size_t(i) + 1]; ++q)
    if (plan.keep_col[size_t(lp.A.idx[size_t(q)])] && ++live > cap) return live;
  return live;
}

// Lower/upper bound on column j from a one-sided row (build_row_affine,
// rule_two_row_variable_elimination.cu:150-200).
bool row_expression(const Lp& lp, const Plan& plan, int i, int j, int max_nnz, double zero_tol, Expr& e,
                    bool& lower) {
  const int live = live_in_row(lp, plan, i, max_nnz);
  if (live < 2 || live > max_nnz || live > kMaxCertified) return false;
  int pivots = 0;
  double pivot = 0.0;
  for (int q = lp.A.ptr[size_t(i)]; q < lp.A.ptr[size_t(i) + 1]; ++q)
    if (plan.keep_col[size_t(lp.A.idx[size_t(q)])] && lp.A.idx[size_t(q)] == j) { ++pivots; pivot = lp.A.val[size_t(q)]; }
  if (pivots != 1 || !std::isfinite(pivot) || std::fabs(pivot) <= zero_tol) return false;
  const double al = plan.AL[size_t(i)], au = plan.AU[size_t(i)];
  double side;
  if (std::isfinite(al) && std::isinf(au) && au > 0.0) { lower = pivot > 0.0; side = al; }
  else if (std::isinf(al) && al < 0.0 && std::isfinite(au)) { lower = pivot < 0.0; side = au; }
  else return false;
  e = Expr{};
  e.constant = side / pivot;
  if (!std::isfinite(e.constant)) return false;
  for (int q = lp.A.ptr[size_t(i)]; q < lp.A.ptr[size_t(i) + 1]; ++q) {
    const int k = lp.A.idx[size_t(q)];
    if (!plan.keep_col[size_t(k)] || k == j) continue;
    if (!add_term(e, k, -lp.A.val[size_t(q)] / pivot, kMaxCertified - 1)) return false;
  }
  return true;
}

bool expr_range(const Expr& e, const Plan& plan, double& lo, double& hi) {
  lo = hi = e.constant;
  for (size_t k = 0; k < e.cols.size(); ++k) {
    const double l = plan.l[size_t(e.cols[k])], u = plan.u[size_t(e.cols[k])], q = e.coeffs[k];
    if (!std::isfinite(l) || !std::isfinite(u) || l > u) return false;
    lo += q >= 0.0 ? q * l : q * u;
    hi += q >= 0.0 ? q * u : q * l;
  }
  return std::isfinite(lo) && std::isfinite(hi);
}

bool max_difference(const Expr& lo_e, const Expr& up_e, const Plan& plan, double& out) {
  Expr d;
  for (size_t k = 0; k < lo_e.cols.size(); ++k)
    if (!add_term(d, lo_e.cols[k], lo_e.coeffs[k], 2 * (kMaxCertified - 1))) return false;
  for (size_t k = 0; k < up_e.cols.size(); ++k)
    if (!add_term(d, up_e.cols[k], -up_e.coeffs[k], 2 * (kMaxCertified - 1))) return false;
  double v = lo_e.constant - up_e.constant;
  for (size_t k = 0; k < d.cols.size(); ++k) {
    const double l = plan.l[size_t(d.cols[k])], u = plan.u[size_t(d.cols[k])];
    if (!std::isfinite(l) || !std::isfinite(u) || l > u) return false;
    v += d.coeffs[k] >= 0.0 ? d.coeffs[k] * u : d.coeffs[k] * l;
  }
  if (!std::isfinite(v)) return false;
  out = v;
  return true;
}

// McCormick row pattern (match_mccormick_row, rule_zero_cost_product_variables.cu:75-150).
bool mccormick_row(const Lp& lp, const Plan& plan, int i, int z, bool& lower, int& e0, int& e1) {
  e0 = e1 = -1;
  const int live = live_in_row(lp, plan, i, 3);
  if (live != 2 && live != 3) return false;
  int pivots = 0;
  double pivot = 0.0;
  for (int q = lp.A.ptr[size_t(i)]; q < lp.A.ptr[size_t(i) + 1]; ++q)
    if (plan.keep_col[size_t(lp.A.idx[size_t(q)])] && lp.A.idx[size_t(q)] == z) { pivot = lp.A.val[size_t(q)]; ++pivots; }
  if (pivots != 1 || !std::isfinite(pivot) || pivot == 0.0) return false;
  const double al = plan.AL[size_t(i)], au = plan.AU[size_t(i)];
  double side;
  if (std::isfinite(al) && std::isinf(au) && au > 0.0) { lower = pivot > 0.0; side = al; }
  else if (std::isinf(al) && al < 0.0 && std::isfinite(au)) { lower = pivot < 0.0; side = au; }
  else return false;
  if (live != (lower ? 3 : 2) || side != (lower ? -pivot : 0.0)) return false;
  int ends = 0;
  for (int q = lp.A.ptr[size_t(i)]; q < lp.A.ptr[size_t(i) + 1]; ++q) {
    const int k = lp.A.idx[size_t(q)];
    if (!plan.keep_col[size_t(k)] || k == z) continue;
    if (lp.A.val[size_t(q)] != -pivot || ends >= 2) return false;
    (ends == 0 ? e0 : e1) = k;
    ++ends;
  }
  return ends == (lower ? 2 : 1) && !(lower && e0 == e1);
}

// Records (before the deletions) and deletions for the selected columns.
void commit_projected(Plan& plan, const Lp& lp, const gpp_params& p, const std::vector<int>& chosen,
                      const std::vector<std::vector<int>>& rows, int K) {
  if (p.record_postsolve_tape) {
    for (int j : chosen) {
      const auto& rr = rows[size_t(j)];
      int lrow = -1;
      double pivot = 0.0, side = 0.0;
      for (int i : rr) {
        int seen = 0;
        double v = 0.0;
        for (int q = lp.A.ptr[size_t(i)]; q < lp.A.ptr[size_t(i) + 1]; ++q)
          if (lp.A.idx[size_t(q)] == j) { v = lp.A.val[size_t(q)]; ++seen; }
        if (seen != 1 || !std::isfinite(v) || v == 0.0) break;
        const double al = plan.AL[size_t(i)], au = plan.AU[size_t(i)];
        const bool lo = std::isfinite(al) && std::isinf(au) && au > 0.0 && v > 0.0;
        const bool up = std::isinf(al) && al < 0.0 && std::isfinite(au) && v < 0.0;
        if (lo || up) { lrow = i; pivot = v; side = lo ? al : au; break; }
      }
      if (lrow < 0) throw std::runtime_error("oracle: projection certificate changed before commit");
      std::vector<int> sup;
      std::vector<double> coef;
      for (int q = lp.A.ptr[size_t(lrow)]; q < lp.A.ptr[size_t(lrow) + 1]; ++q) {
        const int k = lp.A.idx[size_t(q)];
        if (k != j && plan.keep_col[size_t(k)]) { sup.push_back(k); coef.push_back(-lp.A.val[size_t(q)] / pivot); }
      }
      if (K == 3 && sup.size() != 2) throw std::runtime_error("oracle: projection certificate changed before commit");
      std::vector<int> ids{K, j};
      ids.insert(ids.end(), rr.begin(), rr.end());
      const int len = int(sup.size());
      ids.insert(ids.end(), {len, 2, 1, 0, 1, len});
      ids.insert(ids.end(), sup.begin(), sup.end());
      std::vector<double> vals{K == 2 ? plan.l[size_t(j)] : 0.0, side / pivot};
      vals.insert(vals.end(), coef.begin(), coef.end());
      plan.tape.add(FmeCol, ids, vals);
    }
  }
  for (int j : chosen) {
    plan.keep_col[size_t(j)] = 0;
    for (int i : rows[size_t(j)]) plan.keep_row[size_t(i)] = 0;
  }
  plan.has_change = plan.has_row_action = plan.has_col_action = true;
}

// Select candidates whose rows no other candidate uses; threshold on the
// share of the live columns.
template <class Extra>
void select_and_commit(Plan& plan, const Lp& lp, const gpp_params& p, const std::vector<uint8_t>& cand,
                       const std::vector<std::vector<int>>& rows, int K, int live, int min_count, double min_ratio,
                       Extra extra_ok) {
  const int n = lp.n();
  std::vector<int> row_count(size_t(lp.m()), 0);
  for (int j = 0; j < n; ++j)
    if (cand[size_t(j)]) for (int i : rows[size_t(j)]) ++row_count[size_t(i)];
  std::vector<int> chosen;
  for (int j = 0; j < n; ++j) {
    if (!cand[size_t(j)]) continue;
    bool ok = true;
    for (int i : rows[size_t(j)]) ok = ok && row_count[size_t(i)] == 1;
    if (ok && extra_ok(j)) chosen.push_back(j);
  }
  const int count = int(chosen.size());
  const double ratio = double(count) / double(std::max(1, live));
  if (count < std::max(1, min_count) || !(ratio + 1.0e-15 >= min_ratio)) return;
  commit_projected(plan, lp, p, chosen, rows, K);
}

}  // namespace

void rule_two_row_variable_elimination(Plan& plan, const Lp& lp, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (m <= 0 || n <= 0 || lp.A.ptr[size_t(m)] <= 0) return;
  const int max_nnz = std::max(2, std::min(kMaxCertified, p.two_row_variable_elimination_max_row_nnz));
  const double tol = std::max(p.two_row_variable_elimination_safety_tol,
                              std::max(10.0 * p.feasibility_tol, 100.0 * p.zero_tol));
  std::vector<uint8_t> cand(size_t(n), 0);
  std::vector<std::vector<int>> rows(static_cast<size_t>(n), std::vector<int>{});
  int live = 0;
  for (int j = 0; j < n; ++j) {
    if (!plan.keep_col[size_t(j)]) continue;
    ++live;
    const double l = plan.l[size_t(j)], u = plan.u[size_t(j)];
    if (plan.c[size_t(j)] != 0.0 || !std::isfinite(l) || !std::isfinite(u) || !margin_le(l, u, tol)) continue;
    auto rr = kept_rows(lp, plan, j, 2);
    if (rr.empty() || rr[0] == rr[1]) continue;
    Expr e0, e1;
    bool lo0 = false, lo1 = false;
    if (!row_expression(lp, plan, rr[0], j, max_nnz, p.zero_tol, e0, lo0) ||
        !row_expression(lp, plan, rr[1], j, max_nnz, p.zero_tol, e1, lo1) || lo0 == lo1)
      continue;
    const Expr& le = lo0 ? e0 : e1;
    const Expr& ue = lo0 ? e1 : e0;
    double lmin, lmax, umin, umax, diff;
    if (!expr_range(le, plan, lmin, lmax) || !expr_range(ue, plan, umin, umax)) continue;
    if (!margin_le(lmax, u, tol) || !margin_le(l, umin, tol)) continue;
    if (!max_difference(le, ue, plan, diff) || !margin_le(diff, 0.0, tol)) continue;
    cand[size_t(j)] = 1;
    rows[size_t(j)] = rr;
  }
  select_and_commit(plan, lp, p, cand, rows, 2, live, p.two_row_variable_elimination_min_candidates,
                    p.two_row_variable_elimination_min_candidate_ratio, [](int) { return true; });
}

void rule_zero_cost_product_variables(Plan& plan, const Lp& lp, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (m <= 0 || n <= 0 || lp.A.ptr[size_t(m)] <= 0) return;
  std::vector<uint8_t> cand(size_t(n), 0);
  std::vector<std::vector<int>> rows(static_cast<size_t>(n), std::vector<int>{});
  std::vector<int> end0(size_t(n), -1), end1(size_t(n), -1);
  int live = 0;
  for (int z = 0; z < n; ++z) {
    if (!plan.keep_col[size_t(z)]) continue;
    ++live;
    if (plan.c[size_t(z)] != 0.0 || plan.l[size_t(z)] != 0.0 || plan.u[size_t(z)] != 1.0) continue;
    auto rr = kept_rows(lp, plan, z, 3);
    if (rr.empty() || rr[0] == rr[1] || rr[0] == rr[2] || rr[1] == rr[2]) continue;
    int lower_at = -1, nup = 0, ups[2] = {-1, -1};
    bool ok = true;
    int e0[3], e1[3];
    for (int k = 0; k < 3 && ok; ++k) {
      bool lower = false;
      if (!mccormick_row(lp, plan, rr[size_t(k)], z, lower, e0[k], e1[k])) ok = false;
      else if (lower) { if (lower_at >= 0) ok = false; else lower_at = k; }
      else { if (nup >= 2) ok = false; else ups[nup++] = k; }
    }
    if (!ok || lower_at < 0 || nup != 2) continue;
    const int x = e0[lower_at], y = e1[lower_at], ux = e0[ups[0]], uy = e0[ups[1]];
    if (x < 0 || y < 0 || x == y || !((ux == x && uy == y) || (ux == y && uy == x))) continue;
    if (plan.l[size_t(x)] != 0.0 || plan.u[size_t(x)] != 1.0 || plan.l[size_t(y)] != 0.0 || plan.u[size_t(y)] != 1.0)
      continue;
    cand[size_t(z)] = 1;
    rows[size_t(z)] = rr;
    end0[size_t(z)] = x;
    end1[size_t(z)] = y;
  }
  select_and_commit(plan, lp, p, cand, rows, 3, live, p.zero_cost_product_variables_min_candidates,
                    p.zero_cost_product_variables_min_candidate_ratio, [&](int z) {
                      return !cand[size_t(end0[size_t(z)])] && !cand[size_t(end1[size_t(z)])];
                    });
}

}  // namespace oracle

