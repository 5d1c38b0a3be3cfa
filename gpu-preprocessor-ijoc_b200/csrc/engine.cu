// The presolve scheduler: a fixed-point loop of Cleanup, Propagation,
// Aggregation and Parallel phases over a deferred plan that is materialised
// (compacted) at phase boundaries.
//
// Reference: run_gpu_presolve_impl (cpp/src/presolve/gpu_presolve.cu:2081-2645),
// apply_plan_to_working_lp (:1953-2072), capture_cleanup_recovery
// (device_recovery.cu:1011-1027).  The phase machine, the iteration budget,
// the bound-only round limit and the nnz-progress tests follow the reference
// step for step; every rule reports through one status readback.
#include <chrono>
#include <cmath>

#include "engine.cuh"
#include "presolve.hpp"

namespace gpp {

void WorkingLp::free_owned() {
  if (!owns) return;
  free_csr(A);
  free_csr(AT);
  dfree(c); dfree(AL); dfree(AU); dfree(l); dfree(u);
  c = AL = AU = l = u = nullptr;
  owns = false;
}

namespace {

__global__ void fill_u8(uint8_t* p, int n, uint8_t v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

struct Engine {
  const gpp_params& p;
  PresolveOutput& out;
  WorkingLp cur;
  bool terminal = false;
  bool active = false, pending = false;
  Plan plan;
  Stats stats;
  bool stats_dirty = true;
  DBuf<uint8_t> entry_cols;
  DBuf<double> ref_bounds;
  uint32_t* inf_hist = nullptr;   // histogram features (scheduled runs only)
  uint64_t deletion_serial = 0;

  Engine(const gpp_params& params, PresolveOutput& o) : p(params), out(o) {}

  cudaStream_t s() const { return ctx().stream; }

  void init_plan(Plan& pl) {
    const int m = cur.m(), n = cur.n();
    pl.keep_row.alloc(size_t(m), s());
    pl.keep_col.alloc(size_t(n), s());
    GPP_LAUNCH(fill_u8, grid_stride_blocks(m), kThreads, 0, s(), pl.keep_row.p, m, uint8_t(1));
    GPP_LAUNCH(fill_u8, grid_stride_blocks(n), kThreads, 0, s(), pl.keep_col.p, n, uint8_t(1));
    pl.c.alloc(size_t(n), s()); pl.c.copy_from(cur.c, size_t(n));
    pl.l.alloc(size_t(n), s()); pl.l.copy_from(cur.l, size_t(n));
    pl.u.alloc(size_t(n), s()); pl.u.copy_from(cur.u, size_t(n));
    pl.AL.alloc(size_t(m), s()); pl.AL.copy_from(cur.AL, size_t(m));
    pl.AU.alloc(size_t(m), s()); pl.AU.copy_from(cur.AU, size_t(m));
    pl.all_kept = true;
  }
  void prepare() {
    if (active) return;
    plan = Plan{};
    init_plan(plan);
    plan.inf_hist = inf_hist;
    allocate_stats(stats, cur.m(), cur.n());
    entry_cols.alloc(size_t(cur.n()), s());
    stats_dirty = true;
    active = true;
  }
  void refresh() {
    if (stats_dirty) {
      refresh_stats(stats, cur, plan);
      stats_dirty = false;
    }
  }
  int64_t live_nnz() {
    if (!active) return cur.A.nnz;
    refresh();
    return int64_t(read_scalar(stats.live_nnz.p));
  }
  // The live nnz before a phase is used only once the phase is over (its
  // progress test), after the phase's own waits: it is copied to page-locked
  // host memory with no wait of its own, and read when needed (waiting only
  // if no wait has happened since the copy was queued).
  struct LaterCount {
    int64_t value = 0;
    bool pending = false;
    uint64_t queued_at = 0;
  };
  LaterCount live_nnz_later() {
    LaterCount c;
    if (!active) {
      c.value = cur.A.nnz;
      return c;
    }
    refresh();
    check(cudaMemcpyAsync(ctx().host_later, stats.live_nnz.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          s()),
          "live nnz (later)");
    c.pending = true;
    c.queued_at = sync_counter();
    return c;
  }
  int64_t value(LaterCount& c) {
    if (c.pending) {
      if (sync_counter() == c.queued_at) ctx().sync("live_nnz");
      c.value = int64_t(*ctx().host_later);
      c.pending = false;
    }
    return c.value;
  }

  template <class F>
  bool deferred_rule(bool enabled, const char* name, F rule) {
    if (!enabled || terminal) return false;
    const NvtxRange range(name);
    prepare();
    refresh();
    entry_cols.copy_from(plan.keep_col.p, size_t(cur.n()));
    plan.rule_entry_keep_col = entry_cols.p;
    plan.has_change = plan.has_row_action = plan.has_col_action = false;
    plan.has_redundant_row_deletion = plan.has_row_deletion = false;
    plan.obj_delta = 0.0;
    plan.all_kept = false;
    rule();
    out.has_infeasible = plan.has_infeasible;
    out.has_unbounded = plan.has_unbounded;
    terminal = plan.has_infeasible || plan.has_unbounded;
    const bool changed = plan.has_change && !terminal;
    if (changed) {
      if (plan.has_row_deletion || plan.has_col_action) ++deletion_serial;
      cur.obj += plan.obj_delta;
      capture_tape(out.record, plan.tape);
      if (plan.has_col_action)
        append_fixed(out.record, plan.keep_col.p, entry_cols.p, plan.l.p, plan.u.p, cur.n());
      pending = true;
      if (plan.has_row_action || plan.has_col_action) stats_dirty = true;
    } else {
      plan.tape.clear();
    }
    plan.obj_delta = 0.0;
    out.trace.push_back(std::string("rule=") + name + " changed=" + (changed ? "1" : "0"));
    return changed;
  }

  // A rule that a probe of the unchanged plan showed would change nothing:
  // the bookkeeping deferred_rule does for an unchanged rule, without
  // running it.
  bool skipped_rule(bool enabled, const char* name) {
    if (!enabled || terminal) return false;
    prepare();
    refresh();
    out.trace.push_back(std::string("rule=") + name + " changed=0");
    return false;
  }

  // apply_plan_to_working_lp (gpu_presolve.cu:1953-2072).
  void apply(Plan& pl, bool cleanup_captured) {
    const NvtxRange range("materialize");
    Record& r = out.record;
    const int m = cur.m(), n = cur.n();
    // The old -> new maps' kept counts also tell whether the plan removes
    // anything (one readback for both questions).
    DBuf<int32_t> rmap(size_t(std::max(m, 1)), s()), cmap(size_t(std::max(n, 1)), s());
    const auto [m_new, n_new] = build_old_to_new_pair(pl.keep_row.p, m, rmap.p, pl.keep_col.p, n, cmap.p, s());
    if (cur.owns && !pl.has_new_A && m_new == m && n_new == n) {
      capture_tape(r, pl.tape);
      check(cudaMemcpyAsync(cur.c, pl.c.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s()), "commit c");
      check(cudaMemcpyAsync(cur.l, pl.l.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s()), "commit l");
      check(cudaMemcpyAsync(cur.u, pl.u.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s()), "commit u");
      check(cudaMemcpyAsync(cur.AL, pl.AL.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, s()), "commit AL");
      check(cudaMemcpyAsync(cur.AU, pl.AU.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, s()), "commit AU");
      cur.obj += pl.obj_delta;
      return;
    }
    WorkingLp next;
    if (pl.has_new_A) {
      next.A = compact_csr(pl.new_A, rmap.p, m_new, cmap.p, n_new, s());
      next.AT = transpose_csr(next.A, s());
    } else if (cur.AT_sorted()) {
      // A and A^T are compacted back to back; one readback gives both kept
      // counts (equal) and their look-back error words.
      Status st;
      int64_t rec_a = -1, rec_t = -1;
      next.A = compact_csr_queued(cur.A, rmap.p, m_new, cmap.p, n_new, s(), st.d, &rec_a);
      next.AT = compact_csr_queued(cur.AT, cmap.p, n_new, rmap.p, m_new, s(), st.d + 2, &rec_t);
      const int32_t* r = st.read(4);
      compact_csr_finish(next.A, r, rec_a);
      compact_csr_finish(next.AT, r + 2, rec_t);
      if (next.A.nnz != next.AT.nnz) throw std::logic_error("compaction: A and A^T kept different entry counts");
      next.a_sorted = cur.a_sorted;
    } else {
      next.A = compact_csr(cur.A, rmap.p, m_new, cmap.p, n_new, s());
      next.AT = transpose_csr(next.A, s());
      next.a_sorted = cur.a_sorted;
    }
    next.at_sorted = 1;
    next.c = dalloc<double>(size_t(n_new)); gather_by_map(next.c, pl.c.p, cmap.p, n, s());
    next.l = dalloc<double>(size_t(n_new)); gather_by_map(next.l, pl.l.p, cmap.p, n, s());
    next.u = dalloc<double>(size_t(n_new)); gather_by_map(next.u, pl.u.p, cmap.p, n, s());
    next.AL = dalloc<double>(size_t(m_new)); gather_by_map(next.AL, pl.AL.p, rmap.p, m, s());
    next.AU = dalloc<double>(size_t(m_new)); gather_by_map(next.AU, pl.AU.p, rmap.p, m, s());
    next.obj = cur.obj + pl.obj_delta;
    // update_device_recovery (device_recovery.cu:892-975).
    capture_tape(r, pl.tape);
    if (pl.absval) {
      capture_absolute_value(r, std::move(*pl.absval));
      pl.absval.reset();
    }
    if (pl.varpair) {
      capture_variable_pair(r, std::move(*pl.varpair));
      pl.varpair.reset();
    }
    if (!cleanup_captured && n_new != n) append_fixed(r, pl.keep_col.p, nullptr, pl.l.p, pl.u.p, n);
    if (m_new != r.m) {
      DBuf<int32_t> rows(size_t(m_new), s());
      compose_map(rows.p, r.rows.p, rmap.p, m, s());
      r.rows = std::move(rows);
      r.m = m_new;
    }
    if (n_new != r.n) {
      DBuf<int32_t> cols(size_t(n_new), s());
      compose_map(cols.p, r.cols.p, cmap.p, n, s());
      r.cols = std::move(cols);
      r.n = n_new;
    }
    cur.free_owned();
    next.owns = true;
    cur = next;
    invalidate_schedules();
  }

  void materialize(const char* boundary) {
    if (active && pending) {
      apply(plan, true);
      out.trace.push_back(std::string("apply=") + boundary);
    }
    active = pending = false;
    plan = Plan{};
    stats = Stats{};
  }

  template <class F>
  bool materialized_rule(bool enabled, const char* name, F rule) {
    if (!enabled || terminal) return false;
    const NvtxRange range(name);
    Plan pl;
    init_plan(pl);
    rule(pl);
    out.has_infeasible = pl.has_infeasible;
    out.has_unbounded = pl.has_unbounded;
    terminal = pl.has_infeasible || pl.has_unbounded;
    const bool changed = !terminal && pl.has_change;
    if (changed) {
      // A deferred plan still open here (Startup's batch plan when the batch
      // changed nothing) describes the model this rule replaces: retire it,
      // so the next deferred rule starts a fresh plan on the new model.
      if (active) {
        if (pending) throw std::logic_error("materialized rule over a plan with unapplied changes");
        active = false;
        plan = Plan{};
        stats = Stats{};
      }
      apply(pl, false);
      out.trace.push_back(std::string("apply=") + name);
    }
    if (pl.has_new_A) free_csr(pl.new_A);
    return changed;
  }
};

bool good_progress(int64_t before, int64_t after, int64_t d) { return before >= d && after <= before - d; }

}  // namespace

void run_presolve(const gpp_lp& input, const gpp_params& p, PresolveOutput& out, SchedulePolicy* policy,
                  std::vector<RoundRecord>* trace) {
  const NvtxRange range("presolve");
  Engine e(p, out);
  WorkingLp& cur = e.cur;
  cur.A = DevCsr{input.A.rows, input.A.cols, input.A.nnz, input.A.rowPtr, input.A.colVal, input.A.nzVal};
  cur.AT = DevCsr{input.AT.rows, input.AT.cols, input.AT.nnz, input.AT.rowPtr, input.AT.colVal, input.AT.nzVal};
  cur.c = input.c; cur.AL = input.AL; cur.AU = input.AU; cur.l = input.l; cur.u = input.u;
  cur.obj = input.obj_constant;
  cur.owns = false;
  out.original_rows = cur.m();
  out.original_cols = cur.n();
  init_record(out.record, cur.m(), cur.n());
  invalidate_schedules();
  ctx().sync("presolve initialization");
  const auto t0 = std::chrono::steady_clock::now();
  const bool has_time_limit = p.max_time > 0.0 && std::isfinite(p.max_time);
  auto time_exceeded = [&]() {
    return has_time_limit &&
           std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= p.max_time;
  };

  if (p.enable_startup && p.max_iters > 0 && !time_exceeded()) {
    // Startup (gpu_presolve.cu:2361-2454): the structure-specific rules, all
    // off when enable_structure_specific_rules is (:2088-2094).  Column
    // domination, two-row variable elimination and zero-cost product
    // variables share one plan, each seeing the deletions of those before it,
    // and the plan is applied once; then the variable-pair reformulation
    // (:2416-2445) and the absolute-value reformulation, gated by its prefix
    // screen (:2447), each on its own materialised plan.  The phase consumes
    // one iteration (:2453).
    const bool batch = p.enable_structure_specific_rules &&
                       (p.enable_column_domination || p.enable_two_row_variable_elimination ||
                        p.enable_zero_cost_product_variables);
    if (batch && e.deferred_rule(true, "startup_projection_batch", [&] {
          if (p.enable_column_domination) rule_column_domination(e.plan, cur, p);
          if (p.enable_two_row_variable_elimination && !time_exceeded())
            rule_two_row_variable_elimination(e.plan, cur, p);
          if (p.enable_zero_cost_product_variables && !time_exceeded())
            rule_zero_cost_product_variables(e.plan, cur, p);
        }))
      e.materialize("startup");
    if (p.enable_structure_specific_rules && p.enable_piecewise_linear_reformulation_variable_pair && !e.terminal &&
        !time_exceeded())
      e.materialized_rule(true, "startup_piecewise_linear_reformulation_variable_pair",
                          [&](Plan& pl) { rule_variable_pair(pl, cur, p); });
    if (p.enable_structure_specific_rules && p.enable_piecewise_linear_reformulation_absolute_value &&
        !e.terminal && !time_exceeded() && absolute_value_prefix_screen(cur))
      e.materialized_rule(true, "startup_piecewise_linear_reformulation_absolute_value",
                          [&](Plan& pl) { rule_absolute_value(pl, cur, p); });
    ++out.iterations;
  }
  auto deferred = [&](bool enabled, const char* name, auto rule) {
    return !time_exceeded() && e.deferred_rule(enabled, name, rule);
  };
  // Round schedule: `skip` gates rules for the current round (a policy's
  // choice; 0 in the plain loop), `ran` / `changed` record what the gated
  // rules did.
  uint32_t skip = 0, ran = 0, changed_rules = 0;
  auto gate = [&](int rule, bool enabled) {
    const bool run = enabled && !(skip >> rule & 1u);
    if (run) ran |= 1u << rule;
    return run;
  };
  auto note = [&](int rule, bool ch) {
    if (ch) changed_rules |= 1u << rule;
    return ch;
  };
  auto cleanup = [&]() {
    out.trace.push_back("phase=cleanup");
    // The first four rules' first checks run at once on the plan as it stands
    // (one readback instead of four).  While every rule so far has changed
    // nothing the plan is still the probed one, so a rule whose check found
    // nothing is passed over; from the first rule that changes the plan on,
    // the rules run as usual.
    uint32_t may = ~0u;
    const uint32_t probed = (p.enable_infeasible_and_fixed_variables ? kProbeFixed : 0u) |
                            (p.enable_empty_columns ? kProbeEmptyColumns : 0u) |
                            (p.enable_empty_rows ? kProbeEmptyRows : 0u) |
                            (p.enable_singleton_rows ? kProbeSingletonRows : 0u);
    if (probed && !e.terminal && !time_exceeded()) {
      e.prepare();
      e.refresh();
      may = cleanup_probe(e.plan, cur, e.stats, p, probed);
    }
    bool quiet = true;
    auto step = [&](uint32_t bit, bool enabled, const char* name, auto rule) {
      if (quiet && !(may & bit)) return !time_exceeded() && e.skipped_rule(enabled, name);
      const bool changed = deferred(enabled, name, rule);
      quiet = quiet && !changed;
      return changed;
    };
    bool ch = step(kProbeFixed, p.enable_infeasible_and_fixed_variables, "infeasible_and_fixed_variables",
                   [&] { rule_fixed_variables(e.plan, cur, p); });
    ch = step(kProbeEmptyColumns, p.enable_empty_columns, "empty_columns",
              [&] { rule_empty_columns(e.plan, cur, e.stats, p); }) || ch;
    ch = step(kProbeEmptyRows, p.enable_empty_rows, "empty_rows", [&] { rule_empty_rows(e.plan, cur, e.stats, p); }) ||
         ch;
    ch = step(kProbeSingletonRows, p.enable_singleton_rows, "singleton_rows",
              [&] { rule_singleton_rows(e.plan, cur, e.stats, p); }) || ch;
    ch = note(kGateSingletonColumns,
              deferred(gate(kGateSingletonColumns, p.enable_singleton_columns), "singleton_columns",
                       [&] { rule_singleton_columns(e.plan, cur, e.stats, p); })) || ch;
    return ch;
  };
  auto propagation = [&]() {
    out.trace.push_back("phase=propagation");
    bool bounds_changed = false;
    if (gate(kGateBoundStrengthening, p.enable_bound_strengthening) && !e.terminal && !time_exceeded()) {
      e.prepare();
      const int n = cur.n();
      e.ref_bounds.alloc(size_t(2 * std::max(n, 1)), ctx().stream);
      check(cudaMemcpyAsync(e.ref_bounds.p, e.plan.l.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx().stream), "ref l");
      check(cudaMemcpyAsync(e.ref_bounds.p + n, e.plan.u.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx().stream), "ref u");
      e.plan.ref_l = e.ref_bounds.p;
      e.plan.ref_u = e.ref_bounds.p + n;
      bounds_changed = note(kGateBoundStrengthening,
                            e.deferred_rule(true, "bound_strengthening",
                                            [&] { rule_bound_strengthening(e.plan, cur, e.stats, p); }));
    }
    const bool tail = gate(kGateRedundantRowsDualFix, p.enable_infeasible_and_redundant_rows || p.enable_dual_fix);
    bool tail_changed = deferred(tail && p.enable_infeasible_and_redundant_rows, "infeasible_and_redundant_rows",
                                 [&] { rule_redundant_rows(e.plan, cur, e.stats, p); });
    tail_changed = deferred(tail && p.enable_dual_fix, "dual_fix", [&] { rule_dual_fix(e.plan, cur, e.stats, p); }) ||
                   tail_changed;
    note(kGateRedundantRowsDualFix, tail_changed);
    return bounds_changed;
  };

  enum Phase { Cleanup, Propagation, Aggregation, Parallel } phase = Cleanup;
  const int64_t min_dec = 100;
  int bound_only_rounds = 0;
  const int64_t initial_live = p.max_iters > 0 && !e.terminal && !time_exceeded() ? e.live_nnz() : 0;
  const int configured = std::max(1, p.bound_strengthening_max_bound_only_rounds);
  int limit = configured;
  if (p.bound_strengthening_bound_only_nnz_round_budget > 0 && initial_live > 0)
    limit = int(std::min<int64_t>(limit, std::max<int64_t>(1, p.bound_strengthening_bound_only_nnz_round_budget / initial_live)));
  {
    const int64_t m = cur.m(), n = cur.n();
    if (m >= 512 && m <= 2048 && n >= 128 * m && n <= 256 * m && initial_live >= 2048 * m && initial_live <= 8192 * m)
      limit = std::max(limit, std::min(2, configured));
  }
  // Host-side state of the round features.
  const int64_t initial_rows = std::max<int64_t>(1, cur.m());
  const int64_t initial_nnz_all = std::max<int64_t>(1, initial_live);
  int64_t removed_prev = 0, removed_prev2 = 0;
  int round = 0;
  bool last_changed[kGatedRules] = {};
  int last_ran[kGatedRules];
  for (int& r : last_ran) r = -1;
  const bool scheduled = policy || trace;
  DBuf<uint32_t> inf_hist;
  if (scheduled) {
    inf_hist.alloc(8, ctx().stream);
    inf_hist.zero();
    e.inf_hist = inf_hist.p;
    if (e.active) e.plan.inf_hist = inf_hist.p;
  }
  while (p.max_iters > 0 && !e.terminal && !time_exceeded()) {
    if (phase != Cleanup) {
      if (out.iterations >= p.max_iters) { out.stopped_at_iteration_limit = true; break; }
      ++out.iterations;
    }
    // Cleanup does not use the nnz before it (outside traced runs); the other
    // phases read it after their own waits.
    Engine::LaterCount before_count;
    if (scheduled) before_count.value = e.live_nnz();
    else if (phase != Cleanup) before_count = e.live_nnz_later();
    const auto before_nnz = [&]() { return e.value(before_count); };
    RoundRecord rec;
    skip = ran = changed_rules = 0;
    if (scheduled) {
      float* f = rec.features;
      f[int(phase)] = 1.0f;
      f[4] = float(round) / 32.0f;
      f[5] = float(double(before_count.value) / double(initial_nnz_all));
      f[6] = float(double(removed_prev) / double(initial_nnz_all));
      f[7] = float(double(removed_prev2) / double(initial_nnz_all));
      for (int g = 0; g < kGatedRules; ++g) {
        f[8 + g] = last_changed[g] ? 1.0f : 0.0f;
        f[14 + g] = last_ran[g] < 0 ? 1.0f : std::min(1.0f, float(round - last_ran[g]) / 16.0f);
      }
      f[20] = float(bound_only_rounds) / 8.0f;
      f[21] = float(std::log10(double(initial_nnz_all)) / 8.0);
      f[22] = float(1.0 - double(before_count.value) / double(initial_nnz_all));
      f[23] = float(double(cur.m()) / double(initial_rows));
      const std::vector<uint32_t> h = to_host(inf_hist.p, 8);
      for (int side = 0; side < 2; ++side) {
        const double rows = double(h[4 * side] + h[4 * side + 1] + h[4 * side + 2] + h[4 * side + 3]);
        for (int k = 0; k < 4; ++k) f[24 + 4 * side + k] = rows > 0 ? float(double(h[4 * side + k]) / rows) : 0.0f;
      }
      rec.phase = int32_t(phase);
      rec.iteration = out.iterations;
      rec.nnz_before = before_count.value;
      if (policy) {
        bool stop = false;
        skip = policy->decide(f, &stop);
        if (stop) break;
      }
    }
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
      const bool nnz_progress = good_progress(before_nnz(), after, min_dec);
      const bool bound_progress = bounds_changed && bound_only_rounds < limit;
      phase = nnz_progress || bound_progress ? Cleanup : Aggregation;
      if (phase == Aggregation) bound_only_rounds = 0;
    } else if (phase == Aggregation) {
      out.trace.push_back("phase=aggregation");
      if (!time_exceeded() && gate(kGateDoubleton, p.enable_doubleton_equations))
        e.materialized_rule(true, "doubleton_equations", [&](Plan& pl) { rule_doubleton_equations(pl, cur, p); });
      const int64_t after = e.live_nnz();
      const int64_t before = before_nnz();
      note(kGateDoubleton, after < before);
      phase = good_progress(before, after, min_dec) ? Cleanup : Parallel;
    } else {
      out.trace.push_back("phase=parallel");
      bool changed = note(kGateParallelRows,
                          deferred(gate(kGateParallelRows, p.enable_parallel_rows), "parallel_rows",
                                   [&] { rule_parallel_rows(e.plan, cur, e.stats, p); }));
      changed = note(kGateParallelColumns,
                     deferred(gate(kGateParallelColumns, p.enable_parallel_columns), "parallel_columns",
                              [&] { rule_parallel_columns(e.plan, cur, e.stats, p); })) || changed;
      e.materialize("2");
      const int64_t after = e.live_nnz();
      const int64_t before = before_nnz();
      const bool stop_loop = !(changed && good_progress(before, after, min_dec));
      if (scheduled) {
        rec.ran = ran; rec.changed = changed_rules; rec.nnz_after = after;
        if (trace) trace->push_back(rec);
      }
      if (stop_loop) break;
      phase = Cleanup;
      if (scheduled) {
        removed_prev2 = removed_prev;
        removed_prev = before - after;
        for (int g = 0; g < kGatedRules; ++g)
          if (ran >> g & 1u) { last_ran[g] = round; last_changed[g] = (changed_rules >> g & 1u) != 0; }
        ++round;
      }
      continue;
    }
    if (scheduled) {
      const int64_t after = e.live_nnz();
      rec.ran = ran; rec.changed = changed_rules; rec.nnz_after = after;
      if (trace) trace->push_back(rec);
      removed_prev2 = removed_prev;
      removed_prev = before_count.value - after;
      for (int g = 0; g < kGatedRules; ++g)
        if (ran >> g & 1u) { last_ran[g] = round; last_changed[g] = (changed_rules >> g & 1u) != 0; }
      ++round;
    }
  }
  e.materialize("finalize");
  ctx().sync("presolve finalize");
  out.reduced_rows = cur.m();
  out.reduced_cols = cur.n();
  out.reduced_nnz = cur.A.nnz;
  out.obj_constant_delta = cur.obj - input.obj_constant;
  out.elapsed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  out.has_change = cur.owns;
  out.reduced = cur;      // ownership moves to the output when cur.owns
  out.owns_reduced = cur.owns;
  cur.owns = false;
}

}  // namespace gpp
