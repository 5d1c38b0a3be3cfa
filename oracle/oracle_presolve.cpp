// Oracle scheduler, materialisation, recovery record and postsolve: CPU
// restatement of run_gpu_presolve_impl and postsolve_gpu.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <stdexcept>
#include <string>

#include "oracle_rules.hpp"

namespace oracle {

namespace {

inline bool fin(double x) { return std::isfinite(x); }

// globalize (device_recovery.cu:62-183): rewrite local indices to original ones.
void globalize(Tape& t, const std::vector<int>& rows, const std::vector<int>& cols) {
  const int m = int(rows.size()), n = int(cols.size());
  auto mc = [&](int x) { return x >= 0 && x < n ? cols[x] : x; };
  auto mr = [&](int x) { return x >= 0 && x < m ? rows[x] : x; };
  for (int64_t k = 0; k < t.count(); ++k) {
    int* id = t.idx.data() + t.is[k];
    const int64_t sz = t.is[k + 1] - t.is[k];
    switch (t.types[k]) {
      case FixedVariable:
        if (sz) { id[0] = mc(id[0]); for (int64_t q = 1; q < sz; ++q) id[q] = mr(id[q]); }
        break;
      case InfiniteBoundDualFix:
        if (sz >= 3) {
          id[1] = mc(id[1]);
          int64_t q = 3;
          while (q < sz) {
            const int len = id[q++];
            for (int r = 0; r < len && q < sz; ++r, ++q) id[q] = mc(id[q]);
          }
        }
        break;
      case SingletonColumnSubstitution:
        if (sz >= 3) {
          id[0] = mc(id[0]); id[1] = mr(id[1]);
          for (int r = 0; r < id[2] && 3 + r < sz; ++r) id[3 + r] = mc(id[3 + r]);
        }
        break;
      case ParallelColumn:
        if (sz >= 2) { id[0] = mc(id[0]); id[1] = mc(id[1]); }
        break;
      case ParallelRow:
        if (sz >= 2) { id[0] = mr(id[0]); id[1] = mr(id[1]); }
        break;
      case DeletedRow:
        if (sz) { id[0] = mr(id[0]); if (sz >= 2) id[1] = mc(id[1]); }
        break;
      case RowLowerBoundChange: case RowUpperBoundChange: case RowDualShift:
        if (sz) id[0] = mr(id[0]);
        break;
      case VariableBoundChange:
        if (sz) id[0] = mc(id[0]);
        break;
      case RowImpliedBoundChange:
        if (sz >= 2) { id[0] = mc(id[0]); id[1] = mr(id[1]); }
        break;
      case DoubletonEquation:
        if (sz >= 4) {
          id[0] = mc(id[0]); id[1] = mc(id[1]); id[2] = mr(id[2]);
          for (int r = 0; r < id[3] && 4 + r < sz; ++r) id[4 + r] = mr(id[4 + r]);
        }
        break;
      case FmeCol:
        // [K, col, rows[K], terms, L, (orient, len)[L], cols[terms]]
        // (gpu_presolve.cu:1335-1356).
        if (sz >= 4) {
          const int k_rows = id[0];
          id[1] = mc(id[1]);
          for (int r = 0; r < k_rows && 2 + r < sz; ++r) id[2 + r] = mr(id[2 + r]);
          if (3 + k_rows < sz) {
            const int terms = id[2 + k_rows], exprs = id[3 + k_rows];
            const int64_t first = int64_t(4 + k_rows) + 2 * int64_t(exprs);
            for (int q = 0; q < terms && first + q < sz; ++q) id[first + q] = mc(id[first + q]);
          }
        }
        break;
      default:
        throw std::runtime_error("oracle: unknown tape record type");
    }
  }
}

// append_fixed (device_recovery.cu:233-276): columns leaving the model with
// (numerically) equal bounds restore x = (l+u)/2.
void append_fixed(Record& r, const Plan& plan, const std::vector<uint8_t>* prior) {
  for (size_t j = 0; j < plan.keep_col.size(); ++j) {
    if (prior && !(*prior)[j]) continue;
    if (plan.keep_col[j]) continue;
    const double l = plan.l[j], u = plan.u[j];
    if (fin(l) && fin(u) && std::fabs(l - u) <= 1e-9) {
      r.fixed_idx.push_back(r.cols[j]);
      r.fixed_val.push_back(0.5 * (l + u));
    }
  }
}

Csr compact(const Csr& A, const std::vector<int>& row_map, const std::vector<int>& col_map, int m_new,
            int n_new) {
  // compact_csr_by_masks_gpu (gpu_presolve.cu:1793-1930): stable filtering.
  Csr out;
  out.rows = m_new;
  out.cols = n_new;
  out.ptr.assign(size_t(m_new) + 1, 0);
  if (m_new == 0 || n_new == 0) return out;
  for (int i = 0; i < A.rows; ++i) {
    if (row_map[i] < 0) continue;
    for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) {
      const int c = col_map[A.idx[p]];
      if (c < 0) continue;
      out.idx.push_back(c);
      out.val.push_back(A.val[p]);
    }
    out.ptr[size_t(row_map[i]) + 1] = int(out.idx.size());
  }
  for (int i = 0; i < m_new; ++i) out.ptr[i + 1] = std::max(out.ptr[i + 1], out.ptr[i]);
  return out;
}

struct Engine {
  const gpp_params& p;
  Result& res;
  Lp cur;
  bool owns = false;
  bool terminal = false;
  // deferred epoch
  bool active = false, pending = false;
  Plan plan;
  Stats stats;
  std::vector<uint8_t> entry_cols;
  std::vector<double> ref_l, ref_u;
  uint64_t deletion_serial = 0;

  Engine(const gpp_params& params, Result& r) : p(params), res(r) {}

  void prepare() {
    if (active) return;
    plan = Plan{};
    plan.keep_row.assign(cur.m(), 1);
    plan.keep_col.assign(cur.n(), 1);
    plan.c = cur.c; plan.l = cur.l; plan.u = cur.u; plan.AL = cur.AL; plan.AU = cur.AU;
    active = true;
  }
  int64_t live_nnz() {
    if (!active) return cur.A.nnz();
    refresh_stats(stats, cur, plan);
    return stats.live_nnz;
  }
  // capture_cleanup_recovery (device_recovery.cu:1011-1027).
  void capture(bool col_action) {
    globalize(plan.tape, res.record.rows, res.record.cols);
    res.record.tape.append(plan.tape);
    plan.tape = Tape{};
    if (col_action) append_fixed(res.record, plan, &entry_cols);
  }
  template <class F>
  bool deferred_rule(bool enabled, const char* name, F rule) {
    if (!enabled || terminal) return false;
    prepare();
    refresh_stats(stats, cur, plan);
    entry_cols = plan.keep_col;
    plan.rule_entry_keep_col = &entry_cols;
    plan.has_change = plan.has_row_action = plan.has_col_action = false;
    plan.has_redundant_row_deletion = plan.has_row_deletion = false;
    plan.obj_delta = 0.0;
    rule();
    res.summary.has_infeasible = plan.has_infeasible;
    res.summary.has_unbounded = plan.has_unbounded;
    terminal = plan.has_infeasible || plan.has_unbounded;
    const bool changed = plan.has_change && !terminal;
    if (changed) {
      if (plan.has_row_deletion || plan.has_col_action) ++deletion_serial;
      cur.obj += plan.obj_delta;
      capture(plan.has_col_action);
      pending = true;
    }
    plan.obj_delta = 0.0;
    res.trace.push_back(std::string("rule=") + name + " changed=" + (changed ? "1" : "0"));
    return changed;
  }
  // apply_plan_to_working_lp (gpu_presolve.cu:1953-2072).
  void apply(Plan& pl, bool cleanup_captured) {
    std::vector<int> rmap(cur.m(), -1), cmap(cur.n(), -1);
    int m_new = 0, n_new = 0;
    for (int i = 0; i < cur.m(); ++i) if (pl.keep_row[i]) rmap[i] = m_new++;
    for (int j = 0; j < cur.n(); ++j) if (pl.keep_col[j]) cmap[j] = n_new++;
    const Csr& src = pl.has_new_A ? pl.new_A : cur.A;
    Lp next;
    next.A = compact(src, rmap, cmap, m_new, n_new);
    next.AT = transpose(next.A);
    auto gather = [](const std::vector<double>& v, const std::vector<int>& map, int k) {
      std::vector<double> o = std::vector<double>(size_t(k));
      for (size_t i = 0; i < map.size(); ++i) if (map[i] >= 0) o[size_t(map[i])] = v[i];
      return o;
    };
    next.c = gather(pl.c, cmap, n_new);
    next.l = gather(pl.l, cmap, n_new);
    next.u = gather(pl.u, cmap, n_new);
    next.AL = gather(pl.AL, rmap, m_new);
    next.AU = gather(pl.AU, rmap, m_new);
    next.obj = cur.obj + pl.obj_delta;
    // update_device_recovery (device_recovery.cu:892-975).
    Record& r = res.record;
    globalize(pl.tape, r.rows, r.cols);
    r.tape.append(pl.tape);
    pl.tape = Tape{};
    if (!cleanup_captured && n_new != cur.n()) append_fixed(r, pl, nullptr);
    std::vector<int> rows = std::vector<int>(size_t(m_new)), cols = std::vector<int>(size_t(n_new));
    for (int i = 0; i < cur.m(); ++i) if (rmap[i] >= 0) rows[size_t(rmap[i])] = r.rows[i];
    for (int j = 0; j < cur.n(); ++j) if (cmap[j] >= 0) cols[size_t(cmap[j])] = r.cols[j];
    r.rows.swap(rows);
    r.cols.swap(cols);
    cur = std::move(next);
    owns = true;
  }
  void materialize(const char* boundary) {
    if (active && pending) {
      apply(plan, true);
      res.trace.push_back(std::string("apply=") + boundary);
    }
    active = pending = false;
    plan = Plan{};
  }
  template <class F>
  bool materialized_rule(bool enabled, const char* name, F rule) {
    if (!enabled || terminal) return false;
    Plan pl;
    pl.keep_row.assign(cur.m(), 1);
    pl.keep_col.assign(cur.n(), 1);
    pl.c = cur.c; pl.l = cur.l; pl.u = cur.u; pl.AL = cur.AL; pl.AU = cur.AU;
    rule(pl);
    res.summary.has_infeasible = pl.has_infeasible;
    res.summary.has_unbounded = pl.has_unbounded;
    terminal = pl.has_infeasible || pl.has_unbounded;
    const bool changed = !terminal && pl.has_change;
    if (changed) {
      apply(pl, false);
      res.trace.push_back(std::string("apply=") + name);
    }
    return changed;
  }
};

bool good_progress(int64_t before, int64_t after, int64_t d) {
  // has_good_nnz_progress (gpu_presolve.cu:2074-2079).
  return before >= d && after <= before - d;
}

}  // namespace

Result presolve(const Lp& lp, const gpp_params& p) {
  // run_gpu_presolve_impl (gpu_presolve.cu:2081-2645).
  Result res;
  auto& S = res.summary;
  S.original_rows = lp.m();
  S.original_cols = lp.n();
  res.record.m0 = lp.m();
  res.record.n0 = lp.n();
  res.record.rows.resize(size_t(lp.m()));
  res.record.cols.resize(size_t(lp.n()));
  for (int i = 0; i < lp.m(); ++i) res.record.rows[size_t(i)] = i;
  for (int j = 0; j < lp.n(); ++j) res.record.cols[size_t(j)] = j;
  if (!p.enable_presolve) {
    // run_optional_gpu_presolve with presolve off (folding.cu:145-170).
    S.reduced_rows = lp.m();
    S.reduced_cols = lp.n();
    S.reduced_nnz = lp.A.nnz();
    S.presolve_enabled = 0;
    res.reduced = lp;
    return res;
  }
  S.presolve_enabled = 1;
  Engine e(p, res);
  e.cur = lp;
  const auto t0 = std::chrono::steady_clock::now();

  if (p.enable_startup && p.max_iters > 0) {
    // Startup (gpu_presolve.cu:2361-2454): column domination, two-row
    // variable elimination and zero-cost product variables share one plan
    // (each sees the deletions of those before it), applied once before
    // Cleanup; the phase consumes one iteration (:2453).
    const bool batch = p.enable_structure_specific_rules &&
                       (p.enable_column_domination || p.enable_two_row_variable_elimination ||
                        p.enable_zero_cost_product_variables);
    if (batch && e.deferred_rule(true, "startup_projection_batch", [&] {
          if (p.enable_column_domination) rule_column_domination(e.plan, e.cur, p);
          if (p.enable_two_row_variable_elimination) rule_two_row_variable_elimination(e.plan, e.cur, p);
          if (p.enable_zero_cost_product_variables) rule_zero_cost_product_variables(e.plan, e.cur, p);
        }))
      e.materialize("startup");
    ++S.iterations;
  }
  auto cleanup = [&]() {
    res.trace.push_back("phase=cleanup");
    bool ch = e.deferred_rule(p.enable_infeasible_and_fixed_variables, "infeasible_and_fixed_variables",
                              [&] { rule_fixed_variables(e.plan, e.cur, p); });
    ch = e.deferred_rule(p.enable_empty_columns, "empty_columns",
                         [&] { rule_empty_columns(e.plan, e.cur, e.stats, p); }) || ch;
    ch = e.deferred_rule(p.enable_empty_rows, "empty_rows",
                         [&] { rule_empty_rows(e.plan, e.cur, e.stats, p); }) || ch;
    ch = e.deferred_rule(p.enable_singleton_rows, "singleton_rows",
                         [&] { rule_singleton_rows(e.plan, e.cur, e.stats, p); }) || ch;
    ch = e.deferred_rule(p.enable_singleton_columns, "singleton_columns",
                         [&] { rule_singleton_columns(e.plan, e.cur, e.stats, p); }) || ch;
    return ch;
  };
  auto propagation = [&]() {
    res.trace.push_back("phase=propagation");
    bool bounds_changed = false;
    if (p.enable_bound_strengthening && !e.terminal) {
      e.prepare();
      e.ref_l = e.plan.l;
      e.ref_u = e.plan.u;
      e.plan.ref_l = &e.ref_l;
      e.plan.ref_u = &e.ref_u;
      bounds_changed = e.deferred_rule(true, "bound_strengthening",
                                       [&] { rule_bound_strengthening(e.plan, e.cur, e.stats, p); });
    }
    e.deferred_rule(p.enable_infeasible_and_redundant_rows, "infeasible_and_redundant_rows",
                    [&] { rule_redundant_rows(e.plan, e.cur, e.stats, p); });
    e.deferred_rule(p.enable_dual_fix, "dual_fix", [&] { rule_dual_fix(e.plan, e.cur, e.stats, p); });
    return bounds_changed;
  };

  enum Phase { Cleanup, Propagation, Aggregation, Parallel } phase = Cleanup;
  const int64_t min_dec = 100;
  int bound_only_rounds = 0;
  const int64_t initial_live = p.max_iters > 0 && !e.terminal ? e.live_nnz() : 0;
  const int configured = std::max(1, p.bound_strengthening_max_bound_only_rounds);
  int limit = configured;
  if (p.bound_strengthening_bound_only_nnz_round_budget > 0 && initial_live > 0)
    limit = int(std::min<int64_t>(limit, std::max<int64_t>(1, p.bound_strengthening_bound_only_nnz_round_budget / initial_live)));
  {
    const int64_t m = e.cur.m(), n = e.cur.n();
    if (m >= 512 && m <= 2048 && n >= 128 * m && n <= 256 * m && initial_live >= 2048 * m &&
        initial_live <= 8192 * m)
      limit = std::max(limit, std::min(2, configured));
  }
  while (p.max_iters > 0 && !e.terminal) {
    if (phase != Cleanup) {
      if (S.iterations >= p.max_iters) { S.stopped_at_iteration_limit = 1; break; }
      ++S.iterations;
    }
    const int64_t before = e.live_nnz();
    if (phase == Cleanup) {
      const uint64_t ser = e.deletion_serial;
      const bool changed = cleanup();
      if (e.deletion_serial != ser) bound_only_rounds = 0;
      phase = changed ? Cleanup : Propagation;
    } else if (phase == Propagation) {
      const uint64_t ser = e.deletion_serial;
      const bool bounds_changed = propagation();
      bound_only_rounds = e.deletion_serial != ser ? 0 : bound_only_rounds + 1;
      e.materialize("1");
      const int64_t after = e.live_nnz();
      const bool nnz_progress = good_progress(before, after, min_dec);
      const bool bound_progress = bounds_changed && bound_only_rounds < limit;
      phase = nnz_progress || bound_progress ? Cleanup : Aggregation;
      if (phase == Aggregation) bound_only_rounds = 0;
    } else if (phase == Aggregation) {
      res.trace.push_back("phase=aggregation");
      e.materialized_rule(p.enable_doubleton_equations, "doubleton_equations",
                          [&](Plan& pl) { rule_doubleton_equations(pl, e.cur, p); });
      const int64_t after = e.live_nnz();
      phase = good_progress(before, after, min_dec) ? Cleanup : Parallel;
    } else {
      res.trace.push_back("phase=parallel");
      bool changed = e.deferred_rule(p.enable_parallel_rows, "parallel_rows",
                                     [&] { rule_parallel_rows(e.plan, e.cur, e.stats, p); });
      changed = e.deferred_rule(p.enable_parallel_columns, "parallel_columns",
                                [&] { rule_parallel_columns(e.plan, e.cur, e.stats, p); }) || changed;
      e.materialize("2");
      const int64_t after = e.live_nnz();
      if (!(changed && good_progress(before, after, min_dec))) break;
      phase = Cleanup;
    }
  }
  e.materialize("finalize");
  S.reduced_rows = e.cur.m();
  S.reduced_cols = e.cur.n();
  S.reduced_nnz = e.cur.A.nnz();
  S.obj_constant_delta = e.cur.obj - lp.obj;
  S.has_change = e.owns;
  S.owns_reduced_lp = e.owns;
  S.elapsed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  res.reduced = std::move(e.cur);
  return res;
}

// ---------------------------------------------------------------------------
// Postsolve (gpu_postsolve.cu:535-670 and postsolve/*.cuh).

namespace {

constexpr double kTol = 1e-7;
inline bool pfin(double x) { return x > -INFINITY && x < INFINITY; }
inline bool at_lower(double x, double l, double tol) { return pfin(l) && x <= l + tol; }
inline bool at_upper(double x, double u, double tol) { return pfin(u) && x >= u - tol; }
inline double clamp_inf(double x, double lo, double hi) {
  double y = x;
  if (pfin(lo)) y = std::fmax(y, lo);
  if (pfin(hi)) y = std::fmin(y, hi);
  return y;
}

struct Replay {
  double* x; double* y; double* z; std::vector<uint8_t>& got;
  const Lp& M; const Tape& t;

  void fixed_variable(int64_t k, bool primal, bool dual) {
    // replay_fixed_variable (postsolve_fixed_variables.cuh:8-40).
    const int* id = t.idx.data() + t.is[k];
    const double* v = t.val.data() + t.vs[k];
    const int64_t ni = t.is[k + 1] - t.is[k];
    const int col = id[0];
    if (primal) x[col] = v[0];
    if (dual) {
      double zj = v[1];
      for (int64_t q = 1; q < ni; ++q) zj -= v[2 + (q - 1)] * y[id[q]];
      z[col] = zj;
      got[col] = 1;
    }
  }
  void infinite_dual_fix(int64_t k, bool primal, bool dual) {
    // replay_infinite_bound_dual_fix (postsolve_fixed_variables.cuh:42-89).
    const int* id = t.idx.data() + t.is[k];
    const double* v = t.val.data() + t.vs[k];
    const bool pos = id[0] > 0;
    const int col = id[1], nrows = id[2];
    double ext = v[0];
    int64_t ip = 3, vp = 1;
    if (primal) {
      for (int r = 0; r < nrows; ++r) {
        const int len = id[ip];
        double side = v[vp], coeff = 0.0;
        for (int q = 0; q < len; ++q) {
          const int c = id[ip + 1 + q];
          const double a = v[vp + 1 + q];
          if (c == col) coeff = a; else side -= a * x[c];
        }
        const double cand = side / coeff;
        ext = pos ? std::fmax(ext, cand) : std::fmin(ext, cand);
        ip += len + 1;
        vp += len + 1;
      }
      x[col] = ext;
    }
    if (dual) { z[col] = 0.0; got[col] = 1; }
  }
  void singleton_column(int64_t k, bool primal, bool dual) {
    // replay_singleton_column_substitution (postsolve_singleton_columns.cuh:8-50).
    const int* id = t.idx.data() + t.is[k];
    const double* v = t.val.data() + t.vs[k];
    const int ec = id[0], row = id[1], cnt = id[2];
    const double piv = v[0], rhs = v[1], eobj = v[4];
    const bool deleted = v[5] != 0.0;
    double part = 0.0;
    for (int q = 0; q < cnt; ++q) part += v[6 + q] * x[id[3 + q]];
    if (primal) x[ec] = (rhs - part) / piv;
    if (dual && row >= 0) {
      if (deleted) y[row] = eobj / piv; else y[row] += eobj / piv;
    }
    if (dual) {
      z[ec] = deleted ? 0.0 : eobj - piv * y[row];
      got[ec] = 1;
    }
  }
  void run(int64_t k, bool primal, bool dual);
};

// Parallel columns (postsolve_parallel_columns.cuh).
double merged_source_value(double lo, double hi, double tol) {
  if (fin(lo) && fin(hi)) return 0.5 * (lo + hi);
  if (fin(lo)) { if (0.0 > lo + tol) return 0.0; return lo + std::fmax(1.0, std::fabs(lo) * std::fmax(tol, 1.0e-12)); }
  if (fin(hi)) { if (0.0 < hi - tol) return 0.0; return hi - std::fmax(1.0, std::fabs(hi) * std::fmax(tol, 1.0e-12)); }
  return 0.0;
}
double agg_lower(double tl, double sl, double su, double r) {
  if (r > 0.0) { if (fin(tl) && fin(sl)) return tl + r * sl; }
  else if (fin(tl) && fin(su)) return tl + r * su;
  return -INFINITY;
}
double agg_upper(double tu, double sl, double su, double r) {
  if (r > 0.0) { if (fin(tu) && fin(su)) return tu + r * su; }
  else if (fin(tu) && fin(sl)) return tu + r * sl;
  return INFINITY;
}

void Replay::run(int64_t k, bool primal, bool dual) {
  const int type = t.types[k];
  const int* id = t.idx.data() + t.is[k];
  const double* v = t.val.data() + t.vs[k];
  const int64_t ni = t.is[k + 1] - t.is[k], nv = t.vs[k + 1] - t.vs[k];
  const double tol = kTol;
  if (type == ParallelColumn) {
    const int from = id[0], to = id[1];
    const double r = v[0], lo = v[1], hi = v[2], tl = v[3], tu = v[4];
    if (primal) {
      const double yv = x[to], zt = z[to];
      double slo = lo, shi = hi;
      if (fin(tu)) { const double b = (yv - tu) / r; if (r > 0.0) slo = std::fmax(slo, b); else shi = std::fmin(shi, b); }
      if (fin(tl)) { const double b = (yv - tl) / r; if (r > 0.0) shi = std::fmin(shi, b); else slo = std::fmax(slo, b); }
      const double lower = agg_lower(tl, lo, hi, r), upper = agg_upper(tu, lo, hi, r);
      double xf;
      if (zt > tol && fin(lower) && std::fabs(yv - lower) <= tol) xf = r > 0.0 ? lo : hi;
      else if (zt < -tol && fin(upper) && std::fabs(yv - upper) <= tol) xf = r > 0.0 ? hi : lo;
      else xf = merged_source_value(slo, shi, tol);
      x[from] = xf;
      x[to] = yv - r * xf;
    }
    if (dual) { z[from] = r * z[to]; got[from] = 1; }
  } else if (type == DoubletonEquation) {
    // replay_doubleton_equation (postsolve_doubleton_equations.cuh:88-172).
    const int ec = id[0], kc = id[1], row = id[2];
    const double ecoef = v[0], kcoef = v[1], rhs = v[2], eobj = v[9];
    const double alpha = -kcoef / ecoef, beta = rhs / ecoef;
    if (primal) x[ec] = beta + alpha * x[kc];
    if (dual) {
      const double okl = v[5], oku = v[6], nkl = v[7], nku = v[8];
      const double lsrc = nv >= 11 ? v[10] : 0.0, usrc = nv >= 12 ? v[11] : 0.0;
      double zk = 0.0, ze = 0.0;
      const double xk = x[kc], zkh = z[kc];
      if (std::fabs(alpha) <= tol) { zk = zkh; ze = 0.0; }
      else {
        const bool al = pfin(nkl) && xk <= nkl + tol, au = pfin(nku) && xk >= nku - tol;
        if (!al && !au) { zk = 0.0; ze = 0.0; }
        else {
          double src = al ? lsrc : usrc;
          if (src == 0.0) {
            if (al) src = (pfin(okl) && std::fabs(nkl - okl) <= tol) ? 1.0 : 2.0;
            else src = (pfin(oku) && std::fabs(nku - oku) <= tol) ? 1.0 : 2.0;
          }
          if (src == 2.0) { zk = 0.0; ze = zkh / alpha; } else { zk = zkh; ze = 0.0; }
        }
      }
      const bool support = ni >= 4 && nv >= 12;
      double sum_other = 0.0;
      if (support) {
        const int cnt = id[3];
        for (int q = 0; q < cnt; ++q) sum_other += v[12 + q] * y[id[4 + q]];
        y[row] = (eobj - sum_other - ze) / ecoef;
      } else {
        for (int q = M.AT.ptr[ec]; q < M.AT.ptr[ec + 1]; ++q)
          if (M.AT.idx[q] != row) sum_other += M.AT.val[q] * y[M.AT.idx[q]];
        y[row] = (M.c[ec] - sum_other - ze) / ecoef;
      }
      z[kc] = zk; z[ec] = ze; got[kc] = 1; got[ec] = 1;
    }
  } else if (type == SingletonColumnSubstitution) {
    singleton_column(k, primal, dual);
  } else if (type == FixedVariable) {
    fixed_variable(k, primal, dual);
  } else if (type == InfiniteBoundDualFix) {
    infinite_dual_fix(k, primal, dual);
  } else if (type == FmeCol) {
    // replay_projected_column (postsolve_projected_variables.cuh:10-66).
    const int K = id[0], col = id[1], L = id[3 + K];
    int64_t meta = 4 + K, at = 4 + K + 2 * int64_t(L), vp = 0;
    if (primal) {
      double lo = -INFINITY, hi = INFINITY;
      bool has_lo = false, has_hi = false;
      for (int e = 0; e < L; ++e) {
        const int orient = id[meta++], len = id[meta++];
        double cand = v[vp];
        for (int q = 0; q < len; ++q) cand += v[vp + 1 + q] * x[id[at++]];
        if (orient > 0) { lo = std::fmax(lo, cand); has_lo = true; } else { hi = std::fmin(hi, cand); has_hi = true; }
        vp += 1 + len;
      }
      x[col] = has_lo ? lo : (has_hi ? hi : 0.0);
    }
    if (dual) {
      z[col] = 0.0;
      got[col] = 1;
      for (int q = 0; q < K; ++q) y[id[2 + q]] = 0.0;
    }
  } else if (dual && type == RowDualShift) {
    y[id[0]] += v[0];
  } else if (dual && type == ParallelRow && ni >= 2 && nv >= 5) {
    // replay_parallel_row (postsolve_parallel_rows.cuh:170-250).
    const int kept = id[0], del = id[1];
    const double r = v[0], kal = v[1], kau = v[2], dal = v[3], dau = v[4];
    if (std::fabs(r) <= tol) return;
    double dsl = dal * r, dsu = dau * r;
    if (r < 0.0) std::swap(dsl, dsu);
    if (dsl <= kal + tol && kau <= dsu + tol) { y[del] = 0.0; return; }
    auto act = [&](int row) {
      double a = 0.0;
      for (int q = M.A.ptr[row]; q < M.A.ptr[row + 1]; ++q) a += M.A.val[q] * x[M.A.idx[q]];
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
    const double sl = std::fmax(ydl, ypl), sh = std::fmin(ydh, yph);
    if (sl <= sh + tol) {
      const double yd = clamp_inf(0.0, sl, sh);
      y[kept] = y[kept] - yd / r;
      y[del] = yd;
      return;
    }
    // Documented dual split (postsolve_parallel_rows.cuh:120-168).
    const double yb = y[kept];
    double yp = yb, yd = 0.0;
    bool ok;
    if (std::fabs(yb) <= tol) { yp = 0.0; yd = 0.0; ok = true; }
    else {
      const double bl = std::fmax(kal, dsl), bu = std::fmin(kau, dsu);
      if (!(bl <= bu + tol)) { ok = false; }
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
  } else if (dual && type == DeletedRow && ni >= 2 && nv >= 3) {
    // replay_deleted_singleton_row (postsolve_singleton_rows.cuh:8-96).
    const int row = id[0], col = id[1];
    const double oal = v[0], oau = v[1], a = v[2];
    if (std::fabs(a) <= tol) return;
    double g = M.c[col];
    for (int q = M.AT.ptr[col]; q < M.AT.ptr[col + 1]; ++q)
      if (M.AT.idx[q] != row) g -= M.AT.val[q] * y[M.AT.idx[q]];
    const double xj = x[col], zb = z[col], ra = a * xj;
    const bool rl = fin(oal) && ra <= oal + tol, ru = fin(oau) && ra >= oau - tol;
    double lo = -INFINITY, hi = INFINITY;
    if (!(rl && ru)) {
      if (rl) { if (a > 0.0) hi = g; else lo = g; }
      else if (ru) { if (a > 0.0) lo = g; else hi = g; }
      else { lo = g; hi = g; }
    }
    const bool L = at_lower(xj, M.l[col], tol), U = at_upper(xj, M.u[col], tol);
    double zl = lo, zh = hi;
    if (!L && !U) {
      if ((fin(lo) && lo > tol) || (fin(hi) && hi < -tol)) { zl = g; zh = g; } else { zl = 0.0; zh = 0.0; }
    } else if (L && !U) zl = std::fmax(zl, 0.0);
    else if (!L && U) zh = std::fmin(zh, 0.0);
    if (fin(zl) && fin(zh) && zl > zh + tol) return;
    const double zn = clamp_inf(zb, zl, zh);
    z[col] = zn;
    y[row] = (g - zn) / a;
    got[col] = 1;
  } else if (dual && type == RowImpliedBoundChange && ni >= 2) {
    // replay_row_implied_bound_change (postsolve_bound_strengthening.cuh:8-76).
    const int col = id[0], row = id[1];
    if (!got[col]) return;
    const double ol = v[0], ou = v[1], nl = v[2], nu = v[3];
    const bool lc = nl > ol + tol, uc = nu < ou - tol;
    if (lc == uc) return;
    const double ib = lc ? nl : nu, other = lc ? ou : ol;
    const bool other_lower = !lc;
    const double xj = x[col], zj = z[col];
    if (pfin(other) && std::fabs(xj - other) <= tol) {
      const bool ok = other_lower ? (zj >= -tol) : (zj <= tol);
      if (ok) return;
    }
    if (std::fabs(xj - ib) > tol) return;
    double aij = 0.0;
    for (int q = M.A.ptr[row]; q < M.A.ptr[row + 1]; ++q)
      if (M.A.idx[q] == col) { aij = M.A.val[q]; break; }
    if (std::fabs(aij) <= tol) return;
    y[row] += zj / aij;
    for (int q = M.A.ptr[row]; q < M.A.ptr[row + 1]; ++q) {
      const int kc = M.A.idx[q];
      if (kc == col || !got[kc]) continue;
      z[kc] -= (M.A.val[q] / aij) * zj;
    }
    z[col] = 0.0;
    got[col] = 1;
  }
}

}  // namespace

void postsolve(const Result& r, const Lp& M, const double* x_red, const double* y_red,
               const double* z_red, double* x, double* y, double* z) {
  const Record& rec = r.record;
  std::fill(x, x + rec.n0, 0.0);
  std::fill(y, y + rec.m0, 0.0);
  std::fill(z, z + rec.n0, 0.0);
  std::vector<uint8_t> got(size_t(rec.n0), 0);
  for (size_t i = 0; i < rec.cols.size(); ++i) {
    if (x_red) x[rec.cols[i]] = x_red[i];
    if (z_red) z[rec.cols[i]] = z_red[i];
    got[size_t(rec.cols[i])] = 1;
  }
  if (y_red) for (size_t i = 0; i < rec.rows.size(); ++i) y[rec.rows[i]] = y_red[i];
  for (size_t k = 0; k < rec.fixed_idx.size(); ++k) x[rec.fixed_idx[k]] = rec.fixed_val[k];
  Replay rp{x, y, z, got, M, rec.tape};
  const int64_t cnt = rec.tape.count();
  for (int64_t k = cnt - 1; k >= 0; --k) rp.run(k, true, false);
  for (int64_t k = cnt - 1; k >= 0; --k) rp.run(k, false, true);
  // project_column_duals_from_original (gpu_postsolve.cu:355-398).
  std::vector<uint8_t> prot(size_t(rec.n0), 0);
  for (int64_t k = 0; k < cnt; ++k) {
    const int* id = rec.tape.idx.data() + rec.tape.is[k];
    const int t = rec.tape.types[k];
    int a = -1, b = -1;
    if (t == SingletonColumnSubstitution || t == ParallelColumn) a = id[0];
    if (t == DoubletonEquation) { a = id[0]; b = id[1]; }
    if (t == InfiniteBoundDualFix) a = id[1];
    if (a >= 0 && a < rec.n0) prot[size_t(a)] = 1;
    if (b >= 0 && b < rec.n0) prot[size_t(b)] = 1;
  }
  for (int j = 0; j < rec.n0; ++j) {
    if (prot[size_t(j)]) continue;
    double aty = 0.0;
    for (int q = M.AT.ptr[j]; q < M.AT.ptr[j + 1]; ++q) aty += M.AT.val[q] * y[M.AT.idx[q]];
    const double rr = M.c[j] - aty;
    const bool L = at_lower(x[j], M.l[j], kTol), U = at_upper(x[j], M.u[j], kTol);
    double zj;
    if (L && U) zj = rr; else if (!L && !U) zj = 0.0; else if (L) zj = std::fmax(rr, 0.0); else zj = std::fmin(rr, 0.0);
    const double eps = std::fmin(kTol, 1.0e-12);
    if (zj > eps && !fin(M.l[j])) zj = 0.0;
    else if (zj < -eps && !fin(M.u[j])) zj = 0.0;
    z[j] = zj;
  }
}

// Rules not restated yet fail loudly so a parity run can never silently skip them.
#define ORACLE_TODO(name, ...) \
  void name(__VA_ARGS__) { throw std::runtime_error("oracle: " #name " is not restated"); }

}  // namespace oracle
