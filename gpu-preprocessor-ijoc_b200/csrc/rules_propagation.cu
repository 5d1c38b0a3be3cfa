// Propagation rules besides bound strengthening: infeasible / redundant rows
// and lock-based dual fixing.
//
// Reference: rules/rule_infeasible_and_redundant_rows.cu:46-331 and
// rules/rule_dual_fix.cu:203-645 (with the device-resident infinite-bound
// record layout of device_recovery.cu:350-412).
#include "engine.cuh"

namespace gpp {

namespace {

__global__ void redundant_classify(int m, const uint8_t* __restrict__ keep_row, const int32_t* __restrict__ row_nnz,
                                   const double* __restrict__ AL, const double* __restrict__ AU,
                                   const double* __restrict__ mn, const double* __restrict__ mx, double tol,
                                   uint8_t* __restrict__ action, int32_t* __restrict__ status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    uint8_t a = 0;
    if (keep_row[i] && row_nnz[i] > 1) {
      const double al = AL[i], au = AU[i];
      const bool lf = isfinite(al), uf = isfinite(au);
      if (!(lf && uf && fabs(au - al) <= tol)) {
        const double lo = mn[i], hi = mx[i];
        if ((lf && hi < al - tol) || (uf && lo > au + tol)) {
          atomicMax(status + 0, 1);
        } else {
          const bool li = !lf || lo >= al - tol, ui = !uf || hi <= au + tol;
          if (li && ui) { a = 1; atomicMax(status + 1, 1); }
          else if (lf && li) { a = 2; atomicMax(status + 2, 1); }
          else if (uf && ui) { a = 3; atomicMax(status + 3, 1); }
        }
      }
    }
    action[i] = a;
  }
}
__global__ void redundant_apply(int m, const uint8_t* __restrict__ action, uint8_t* __restrict__ keep_row,
                                double* __restrict__ AL, double* __restrict__ AU) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const uint8_t a = action[i];
    if (a == 1) keep_row[i] = 0;
    else if (a == 2) AL[i] = -INFINITY;
    else if (a == 3) AU[i] = INFINITY;
  }
}

// _kernel_dual_fix_candidates (rule_dual_fix.cu:205-309).
__global__ void dual_fix_candidates(int n, const uint8_t* __restrict__ keep_col, const uint8_t* __restrict__ keep_row,
                                    const double* __restrict__ c, const double* __restrict__ l,
                                    const double* __restrict__ u, const double* __restrict__ AL,
                                    const double* __restrict__ AU, const offset_t* __restrict__ at_ptr,
                                    const int32_t* __restrict__ at_idx, const double* __restrict__ at_val,
                                    double zt, double bound_tol, int max_degree, const int32_t* __restrict__ col_nnz,
                                    uint8_t* __restrict__ fixed, uint8_t* __restrict__ inf_fix,
                                    double* __restrict__ fval, double* __restrict__ contrib,
                                    int32_t* __restrict__ status) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    fixed[j] = 0; inf_fix[j] = 0; fval[j] = 0.0; contrib[j] = 0.0;
    if (!keep_col[j]) continue;
    const double lj = l[j], uj = u[j];
    if (lj > uj + bound_tol) { atomicMax(status + 0, 1); continue; }
    const double cj = c[j];
    if (fabs(cj) > zt && col_nnz[j] > max_degree) continue;
    bool down = false, up = false;
    for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p) {
      const int row = at_idx[p];
      if (!keep_row[row]) continue;
      const double a = at_val[p];
      if (a > zt) { down = down || isfinite(AL[row]); up = up || isfinite(AU[row]); }
      else if (a < -zt) { down = down || isfinite(AU[row]); up = up || isfinite(AL[row]); }
      if (down && up) break;
    }
    bool f = false, fi = false;
    double v = 0.0;
    if (cj > zt) {
      if (!down) { if (isfinite(lj)) { v = lj; f = true; } else { atomicMax(status + 0, 2); continue; } }
    } else if (cj < -zt) {
      if (!up) { if (isfinite(uj)) { v = uj; f = true; } else { atomicMax(status + 0, 2); continue; } }
    } else if (fabs(cj) <= zt) {
      if (!down) { f = true; if (isfinite(lj)) v = lj; else { v = -INFINITY; fi = true; } }
      else if (!up) { f = true; if (isfinite(uj)) v = uj; else { v = INFINITY; fi = true; } }
    }
    if (f) {
      fixed[j] = 1; inf_fix[j] = fi; fval[j] = v; contrib[j] = fi ? 0.0 : cj * v;
      atomicMax(status + 1, 1);
      if (fi) atomicMax(status + 2, 1);
    }
  }
}
__global__ void finite_fixed_mask(int n, const uint8_t* __restrict__ fixed, const uint8_t* __restrict__ inf_fix,
                                  uint8_t* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    out[j] = fixed[j] && !inf_fix[j];
}
__global__ void dual_fix_row_remove(int n, const uint8_t* __restrict__ fixed, const uint8_t* __restrict__ inf_fix,
                                    const uint8_t* __restrict__ keep_row, const offset_t* __restrict__ at_ptr,
                                    const int32_t* __restrict__ at_idx, uint8_t* __restrict__ remove,
                                    int32_t* __restrict__ status) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (!(fixed[j] && inf_fix[j])) continue;
    for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p)
      if (keep_row[at_idx[p]]) { remove[at_idx[p]] = 1; atomicMax(status + 3, 1); }
  }
}
// InfiniteBoundDualFix record sizes: 1 record per column, 3 + rows + entries
// indices and 1 + rows + entries values (entries restricted to the entry domain).
__global__ void infinite_sizes(int n, const uint8_t* __restrict__ fixed, const uint8_t* __restrict__ inf_fix,
                               const uint8_t* __restrict__ keep_row, const uint8_t* __restrict__ entry,
                               const offset_t* __restrict__ a_ptr, const int32_t* __restrict__ a_idx,
                               const offset_t* __restrict__ at_ptr, const int32_t* __restrict__ at_idx,
                               int64_t* __restrict__ recs, int64_t* __restrict__ sizes) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const bool sel = fixed[j] && inf_fix[j];
    int64_t size = 0;
    if (sel)
      for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p) {
        const int row = at_idx[p];
        if (!keep_row[row]) continue;
        ++size;
        for (offset_t q = a_ptr[row]; q < a_ptr[row + 1]; ++q) size += entry[a_idx[q]] != 0;
      }
    recs[j] = sel;
    sizes[j] = size;
  }
}
__global__ void infinite_pack(int n, const uint8_t* __restrict__ fixed, const uint8_t* __restrict__ inf_fix,
                              const double* __restrict__ fval, const uint8_t* __restrict__ keep_row,
                              const uint8_t* __restrict__ entry, const double* __restrict__ l,
                              const double* __restrict__ u, const double* __restrict__ AL,
                              const double* __restrict__ AU, const offset_t* __restrict__ a_ptr,
                              const int32_t* __restrict__ a_idx, const double* __restrict__ a_val,
                              const offset_t* __restrict__ at_ptr, const int32_t* __restrict__ at_idx,
                              const int64_t* __restrict__ rpos, const int64_t* __restrict__ spos,
                              int32_t* __restrict__ types, int64_t* __restrict__ is, int64_t* __restrict__ vs,
                              int32_t* __restrict__ idx, double* __restrict__ val) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (j == 0) { is[0] = 0; vs[0] = 0; }
    if (!(fixed[j] && inf_fix[j])) continue;
    const int64_t k = rpos[j], base = spos[j];
    int64_t ip = base + 3 * k, vp = base + k;
    const bool pos = fval[j] > 0;
    types[k] = 1;  // InfiniteBoundDualFix
    idx[ip++] = pos ? 1 : -1;
    idx[ip++] = j;
    const int64_t count_pos = ip++;
    val[vp++] = pos ? l[j] : u[j];
    int active = 0;
    for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p) {
      const int row = at_idx[p];
      if (!keep_row[row]) continue;
      ++active;
      const int64_t header = ip++;
      int len = 0;
      val[vp++] = isfinite(AL[row]) ? AL[row] : AU[row];
      for (offset_t q = a_ptr[row]; q < a_ptr[row + 1]; ++q) {
        if (!entry[a_idx[q]]) continue;
        ++len;
        idx[ip++] = a_idx[q];
        val[vp++] = a_val[q];
      }
      idx[header] = len;
    }
    idx[count_pos] = active;
    is[k + 1] = ip;
    vs[k + 1] = vp;
  }
}
__global__ void dual_fix_apply(int n, int m, const uint8_t* __restrict__ fixed, const double* __restrict__ fval,
                               const uint8_t* __restrict__ remove, const double* __restrict__ shift,
                               uint8_t* __restrict__ keep_col, uint8_t* __restrict__ keep_row,
                               double* __restrict__ l, double* __restrict__ u, double* __restrict__ AL,
                               double* __restrict__ AU) {
  const int top = n > m ? n : m;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < top; k += gridDim.x * blockDim.x) {
    if (k < n && fixed[k]) { l[k] = fval[k]; u[k] = fval[k]; keep_col[k] = 0; }
    if (k < m) {
      AL[k] -= shift[k];
      AU[k] -= shift[k];
      if (remove[k]) keep_row[k] = 0;
    }
  }
}

}  // namespace

void rule_redundant_rows(Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m();
  if (m == 0) return;
  auto s = ctx().stream;
  DBuf<double> mn(size_t(m), s), mx(size_t(m), s);
  DBuf<uint8_t> action(size_t(m), s);
  row_plain_minmax(lp.A, plan.l.p, plan.u.p, plan.keep_row.p, plan.keep_col.p, stats.row_nnz.p, mn.p, mx.p, s);
  Status st;
  st.clear(4);
  GPP_LAUNCH(redundant_classify, grid_stride_blocks(m), kThreads, 0, s, m, plan.keep_row.p, stats.row_nnz.p,
             plan.AL.p, plan.AU.p, mn.p, mx.p, p.bound_tol, action.p, st.d);
  const int32_t* f = st.read(4);
  if (f[0]) { plan.has_infeasible = true; return; }
  if (!f[1] && !f[2] && !f[3]) return;
  const bool deleted = f[1] != 0;
  GPP_LAUNCH(redundant_apply, grid_stride_blocks(m), kThreads, 0, s, m, action.p, plan.keep_row.p, plan.AL.p,
             plan.AU.p);
  plan.has_row_action = true;
  plan.has_redundant_row_deletion = plan.has_redundant_row_deletion || deleted;
  plan.has_row_deletion = plan.has_row_deletion || deleted;
  plan.has_change = true;
}

void rule_dual_fix(Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int n = lp.n(), m = lp.m();
  if (n == 0) return;
  auto s = ctx().stream;
  DBuf<uint8_t> fixed(size_t(n), s), inf_fix(size_t(n), s), finite(size_t(n), s), remove(size_t(std::max(m, 1)), s);
  DBuf<double> fval(size_t(n), s), contrib(size_t(n), s), shift(size_t(std::max(m, 1)), s);
  Status st;
  st.clear(4);
  GPP_LAUNCH(dual_fix_candidates, grid_stride_blocks(n), kThreads, 0, s, n, plan.keep_col.p, plan.keep_row.p,
             plan.c.p, plan.l.p, plan.u.p, plan.AL.p, plan.AU.p, lp.AT.ptr, lp.AT.idx, lp.AT.val, p.zero_tol,
             p.bound_tol, p.dual_fix_max_nonzero_cost_col_degree, stats.col_nnz.p, fixed.p, inf_fix.p, fval.p,
             contrib.p, st.d);
  const int32_t* f = st.read(3);
  if (f[0] == 1) { plan.has_infeasible = true; return; }
  if (f[0] == 2) { plan.has_unbounded = true; return; }
  if (!f[1]) return;
  const bool any_inf = f[2] != 0;
  GPP_LAUNCH(finite_fixed_mask, grid_stride_blocks(n), kThreads, 0, s, n, fixed.p, inf_fix.p, finite.p);
  if (m) {
    row_gather_shift(lp.A, lp.AT, plan.keep_row.p, finite.p, fval.p, nullptr, shift.p, s);
    remove.zero();
  }
  GPP_LAUNCH(dual_fix_row_remove, grid_stride_blocks(n), kThreads, 0, s, n, fixed.p, inf_fix.p, plan.keep_row.p,
             lp.AT.ptr, lp.AT.idx, remove.p, st.d);
  const bool row_changed = st.read(4)[3] != 0;
  if (p.record_postsolve_tape && any_inf) {
    DBuf<int64_t> rc(size_t(n) + 1, s), sz(size_t(n) + 1, s), rpos(size_t(n) + 1, s), spos(size_t(n) + 1, s);
    GPP_LAUNCH(infinite_sizes, grid_stride_blocks(n), kThreads, 0, s, n, fixed.p, inf_fix.p, plan.keep_row.p,
               plan.rule_entry_keep_col, lp.A.ptr, lp.A.idx, lp.AT.ptr, lp.AT.idx, rc.p, sz.p);
    exclusive_scan_i64(rc.p, rpos.p, n, s);
    exclusive_scan_i64(sz.p, spos.p, n, s);
    const auto [recs, size] = read_scalars(rpos.p + n, spos.p + n);
    if (recs) {
      PostsolveSegment seg = make_segment(recs, size + 3 * recs, size + recs);
      GPP_LAUNCH(infinite_pack, grid_stride_blocks(n), kThreads, 0, s, n, fixed.p, inf_fix.p, fval.p, plan.keep_row.p,
                 plan.rule_entry_keep_col, plan.l.p, plan.u.p, plan.AL.p, plan.AU.p, lp.A.ptr, lp.A.idx, lp.A.val,
                 lp.AT.ptr, lp.AT.idx, rpos.p, spos.p, seg.types.p, seg.is.p, seg.vs.p, seg.idx.p, seg.val.p);
      plan.tape.push_back(std::move(seg));
    }
  }
  GPP_LAUNCH(dual_fix_apply, grid_stride_blocks(std::max(n, m)), kThreads, 0, s, n, m, fixed.p, fval.p, remove.p,
             shift.p, plan.keep_col.p, plan.keep_row.p, plan.l.p, plan.u.p, plan.AL.p, plan.AU.p);
  plan.obj_delta += domain_objective(contrib.p, plan.rule_entry_keep_col, n, s);
  plan.has_row_action = plan.has_row_action || row_changed;
  plan.has_col_action = plan.has_change = true;
}

}  // namespace gpp
