// Cleanup rules: infeasible/fixed variables, empty columns, empty rows and
// singleton rows.  Each rule works on the deferred plan (keep masks plus the
// working copies of c, l, u, AL, AU) over the physical A / A^T, and reports
// through one status block read back once per rule.
//
// Reference: rules/rule_infeasible_and_fixed_variables.cu:65-348,
// rules/empty_rows_and_columns/columns.cu:64-249, rows.cu:26-121,
// rules/rule_singleton_rows.cu:76-275.
#include "engine.cuh"

namespace gpp {

namespace {


// Rows touched by a selected column (with positive radius in radius mode).
__global__ void mark_touched_rows(int n, const offset_t* __restrict__ at_ptr, const int32_t* __restrict__ at_idx,
                                  const uint8_t* __restrict__ selected, const double* __restrict__ radius,
                                  uint8_t* __restrict__ touched) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (!selected[j] || (radius && !(radius[j] > 0.0))) continue;
    for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p) touched[at_idx[p]] = 1;
  }
}

// Kept touched rows are listed; every other row's sum is 0.
__global__ void list_touched_rows(int m, const uint8_t* __restrict__ keep_row, const uint8_t* __restrict__ touched,
                                  int32_t* __restrict__ list, int32_t* counter, double* __restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  const int top = (m + stride - 1) / stride * stride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < top; i += stride) {
    const bool take = i < m && keep_row[i] && touched[i];
    if (i < m && !take) out[i] = 0.0;
    const int at = block_append(counter, take);
    if (take) list[at] = i;
  }
}

// Row sums over selected columns, added in stored (ascending column) order:
// one warp per listed row computes 32 terms at a time and lane 0 adds them in
// order, so long rows no longer serialise on one thread's loads.
__global__ void row_gather_kernel(const int32_t* __restrict__ list, const int32_t* __restrict__ count,
                                  const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                  const double* __restrict__ val, const uint8_t* __restrict__ selected,
                                  const double* __restrict__ value, const double* __restrict__ radius,
                                  double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int k = *count;
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < k; w += warps) {
    const int i = list[w];
    double acc = 0.0;
    for (offset_t chunk = ptr[i]; chunk < ptr[i + 1]; chunk += 32) {
      const offset_t p = chunk + lane;
      double term = 0.0;
      bool has = false;
      if (p < ptr[i + 1]) {
        const int j = __ldcs(idx + p);
        if (selected[j]) {
          if (radius) {
            if (radius[j] > 0.0) { has = true; term = fabs(__ldcs(val + p)) * radius[j]; }
          } else {
            has = true;
            term = __ldcs(val + p) * value[j];
          }
        }
      }
      const unsigned hv = __ballot_sync(0xffffffffu, has);
      if (!hv) continue;
      for (int q = 0; q < 32; ++q) {
        const double v = __shfl_sync(0xffffffffu, term, q);
        if (hv >> q & 1u) acc += v;
      }
    }
    if (lane == 0) out[i] = acc;
  }
}

__global__ void mask_contrib(int n, const double* __restrict__ contrib, const uint8_t* __restrict__ entry,
                             double* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    out[j] = entry && !entry[j] ? 0.0 : contrib[j];
}

// --- infeasible / fixed variables ------------------------------------------
__global__ void fixed_candidates(int n, const uint8_t* __restrict__ keep_col, const double* __restrict__ l,
                                 const double* __restrict__ u, const double* __restrict__ c, double bound_tol,
                                 uint8_t* __restrict__ fixed, double* __restrict__ fval,
                                 double* __restrict__ contrib, double* __restrict__ radius, int32_t* __restrict__ any) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    uint8_t f = 0;
    double v = 0.0, cb = 0.0, rad = 0.0;
    if (keep_col[j]) {
      const double lj = l[j], uj = u[j];
      if (isfinite(lj) && isfinite(uj) && lj <= uj && uj - lj <= bound_tol) {
        v = lj + 0.5 * (uj - lj);
        rad = fmax(v - lj, uj - v);
        f = 1;
        cb = c[j] * v;
      }
    }
    fixed[j] = f; fval[j] = v; contrib[j] = cb; radius[j] = rad;
    if (f) *any = 1;
  }
}
__global__ void fixed_filter(int n, const offset_t* __restrict__ at_ptr, const int32_t* __restrict__ at_idx,
                             const uint8_t* __restrict__ keep_row, const double* __restrict__ l,
                             const double* __restrict__ u, const double* __restrict__ row_error, double budget,
                             uint8_t* __restrict__ fixed, double* __restrict__ contrib, int32_t* __restrict__ status) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (!fixed[j]) continue;
    bool keep_fix = true;
    if (l[j] != u[j])
      for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p) {
        const int row = at_idx[p];
        if (keep_row[row] && !(row_error[row] <= budget)) { keep_fix = false; break; }
      }
    if (!keep_fix) { fixed[j] = 0; contrib[j] = 0.0; }
    else atomicAdd(status, 1);
  }
}
__global__ void fixed_apply(int n, int m, const uint8_t* __restrict__ fixed, const double* __restrict__ fval,
                            const double* __restrict__ shift, uint8_t* __restrict__ keep_col, double* __restrict__ l,
                            double* __restrict__ u, double* __restrict__ AL, double* __restrict__ AU) {
  const int top = n > m ? n : m;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < top; j += gridDim.x * blockDim.x) {
    if (j < n && fixed[j]) { l[j] = fval[j]; u[j] = fval[j]; keep_col[j] = 0; }
    if (j < m) { AL[j] -= shift[j]; AU[j] -= shift[j]; }
  }
}

// --- empty columns -----------------------------------------------------------
__global__ void empty_columns_classify(int n, const uint8_t* __restrict__ keep_col, const uint8_t* __restrict__ empty,
                                       const double* __restrict__ c, const double* __restrict__ l,
                                       const double* __restrict__ u, double bound_tol, double zero_tol,
                                       uint8_t* __restrict__ fixed, double* __restrict__ fval,
                                       double* __restrict__ contrib, int32_t* __restrict__ status) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    fixed[j] = 0; fval[j] = 0.0; contrib[j] = 0.0;
    if (!(keep_col[j] && empty[j])) continue;
    const double cj = c[j], lj = l[j], uj = u[j];
    if (lj > uj + bound_tol) { atomicMax(status + 0, 1); continue; }
    if ((cj > zero_tol && !isfinite(lj)) || (cj < -zero_tol && !isfinite(uj))) { atomicMax(status + 1, 1); continue; }
    double v = 0.0;
    if (cj > zero_tol) v = lj;
    else if (cj < -zero_tol) v = uj;
    else if (isfinite(lj)) v = lj;
    else if (isfinite(uj)) v = uj;
    fixed[j] = 1; fval[j] = v; contrib[j] = cj * v;
    atomicMax(status + 2, 1);
  }
}
__global__ void fix_columns(int n, const uint8_t* __restrict__ fixed, const double* __restrict__ fval,
                            uint8_t* __restrict__ keep_col, double* __restrict__ l, double* __restrict__ u) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    if (fixed[j]) { l[j] = fval[j]; u[j] = fval[j]; keep_col[j] = 0; }
}

// --- empty rows ----------------------------------------------------------------
__global__ void empty_rows_kernel(int m, uint8_t* __restrict__ keep_row, const int32_t* __restrict__ row_nnz,
                                  const double* __restrict__ AL, const double* __restrict__ AU, double tol,
                                  int32_t* __restrict__ status, int apply) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    if (!(keep_row[i] && row_nnz[i] == 0)) continue;
    const bool feasible = AL[i] <= tol && AU[i] >= -tol;
    if (!apply) atomicMax(status + (feasible ? 1 : 0), 1);
    else if (feasible) keep_row[i] = 0;
  }
}

// --- singleton rows -----------------------------------------------------------
__global__ void singleton_row_bounds(int m, int n, const uint8_t* __restrict__ keep_row,
                                     const uint8_t* __restrict__ singleton, const int32_t* __restrict__ scol,
                                     const double* __restrict__ sval, const double* __restrict__ AL,
                                     const double* __restrict__ AU, double zero_tol, double* cand_l, double* cand_u,
                                     uint8_t* __restrict__ remove) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    remove[i] = 0;
    if (!(keep_row[i] && singleton[i])) continue;
    const int col = scol[i];
    const double a = sval[i];
    if (!(col >= 0 && col < n && fabs(a) > zero_tol)) continue;
    const double lo = AL[i], hi = AU[i];
    red_max_f64(&cand_l[col], a > 0.0 ? lo / a : hi / a);
    red_min_f64(&cand_u[col], a > 0.0 ? hi / a : lo / a);
    remove[i] = 1;
  }
}
__global__ void singleton_rows_check(int m, int n, const double* __restrict__ cand_l, const double* __restrict__ cand_u,
                                     const double* __restrict__ l, const double* __restrict__ u,
                                     const uint8_t* __restrict__ remove, double tol, int32_t* __restrict__ status) {
  const int top = n > m ? n : m;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < top; j += gridDim.x * blockDim.x) {
    if (j < n) {
      if (cand_l[j] > cand_u[j] + tol) atomicMax(status + 0, 1);
      if (cand_l[j] != l[j] || cand_u[j] != u[j]) atomicMax(status + 2, 1);
    }
    if (j < m && remove[j]) atomicMax(status + 1, 1);
  }
}
__global__ void singleton_rows_commit(int m, int n, const uint8_t* __restrict__ remove, uint8_t* __restrict__ keep_row) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    if (remove[i]) keep_row[i] = 0;
}

}  // namespace

void row_gather_shift(const DevCsr& A, const DevCsr& AT, const uint8_t* keep_row, const uint8_t* selected,
                      const double* value, const double* radius, double* out, cudaStream_t s) {
  DBuf<uint8_t> touched(size_t(std::max(A.rows, 1)), s);
  DBuf<int32_t> list(size_t(std::max(A.rows, 1)), s), count(1, s);
  touched.zero();
  count.zero();
  GPP_LAUNCH(mark_touched_rows, grid_stride_blocks(AT.rows), kThreads, 0, s, AT.rows, AT.ptr, AT.idx, selected, radius,
             touched.p);
  GPP_LAUNCH(list_touched_rows, grid_stride_blocks(A.rows), kThreads, 0, s, A.rows, keep_row, touched.p, list.p,
             count.p, out);
  GPP_LAUNCH(row_gather_kernel, kNumSMs * 16, kThreads, 0, s, list.p, count.p, A.ptr, A.idx, A.val, selected, value,
             radius, out);
}

double domain_objective(const double* contrib, const uint8_t* entry_keep, int32_t n, cudaStream_t s) {
  // sum_cleanup_domain (cleanup_support.cuh:13-31): the sum over the rule's
  // entry domain, with the canonical deterministic reduction.
  if (n <= 0) return 0.0;
  DBuf<double> masked(size_t(n), s);
  GPP_LAUNCH(mask_contrib, grid_stride_blocks(n), kThreads, 0, s, n, contrib, entry_keep, masked.p);
  return det_sum(masked.p, n, s);
}

uint32_t cleanup_probe(const Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p, uint32_t rules) {
  // The first-stage detections of the four rules below, on the current plan,
  // with one readback.  Each is the kernel its rule launches first and writes
  // only scratch and status words; a rule whose detection finds nothing
  // (no candidate, no infeasibility) returns without touching the plan.
  if (plan.has_infeasible || plan.has_unbounded) return rules;
  const int n = lp.n(), m = lp.m();
  auto s = ctx().stream;
  Status st;
  st.clear(16);
  DBuf<uint8_t> fixed(size_t(std::max(n, 1)), s), remove(size_t(std::max(m, 1)), s);
  DBuf<double> fval(size_t(std::max(n, 1)), s), contrib(size_t(std::max(n, 1)), s), radius(size_t(std::max(n, 1)), s);
  DBuf<double> cl, cu;
  if ((rules & kProbeFixed) && n > 0)
    GPP_LAUNCH(fixed_candidates, grid_stride_blocks(n), kThreads, 0, s, n, plan.keep_col.p, plan.l.p, plan.u.p,
               plan.c.p, p.bound_tol, fixed.p, fval.p, contrib.p, radius.p, st.d + 1);
  if ((rules & kProbeEmptyColumns) && n > 0)
    GPP_LAUNCH(empty_columns_classify, grid_stride_blocks(n), kThreads, 0, s, n, plan.keep_col.p, stats.empty_col.p,
               plan.c.p, plan.l.p, plan.u.p, p.bound_tol, p.zero_tol, fixed.p, fval.p, contrib.p, st.d + 4);
  if ((rules & kProbeEmptyRows) && m > 0)
    GPP_LAUNCH(empty_rows_kernel, grid_stride_blocks(m), kThreads, 0, s, m, plan.keep_row.p, stats.row_nnz.p,
               plan.AL.p, plan.AU.p, p.feasibility_tol, st.d + 8, 0);
  if ((rules & kProbeSingletonRows) && m > 0) {
    cl.alloc(size_t(std::max(n, 1)), s);
    cu.alloc(size_t(std::max(n, 1)), s);
    cl.copy_from(plan.l.p, size_t(n));
    cu.copy_from(plan.u.p, size_t(n));
    GPP_LAUNCH(singleton_row_bounds, grid_stride_blocks(m), kThreads, 0, s, m, n, plan.keep_row.p,
               stats.singleton_row.p, stats.srow_col.p, stats.srow_val.p, plan.AL.p, plan.AU.p, p.zero_tol, cl.p,
               cu.p, remove.p);
    GPP_LAUNCH(singleton_rows_check, grid_stride_blocks(std::max(m, n)), kThreads, 0, s, m, n, cl.p, cu.p, plan.l.p,
               plan.u.p, remove.p, p.bound_tol, st.d + 12);
  }
  const int32_t* f = st.read(16);
  uint32_t act = 0;
  if ((rules & kProbeFixed) && n > 0 && f[1] != 0) act |= kProbeFixed;
  if ((rules & kProbeEmptyColumns) && n > 0 && (f[4] | f[5] | f[6]) != 0) act |= kProbeEmptyColumns;
  if ((rules & kProbeEmptyRows) && m > 0 && (f[8] | f[9]) != 0) act |= kProbeEmptyRows;
  if ((rules & kProbeSingletonRows) && m > 0 && (f[12] | f[13] | f[14]) != 0) act |= kProbeSingletonRows;
  return act;
}

void rule_fixed_variables(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int n = lp.n(), m = lp.m();
  if (n == 0) return;
  auto s = ctx().stream;
  DBuf<uint8_t> fixed(size_t(n), s);
  DBuf<double> fval(size_t(n), s), contrib(size_t(n), s), radius(size_t(n), s), row_err(size_t(m), s),
      shift(size_t(m), s);
  Status st;
  st.clear(4);
  GPP_LAUNCH(fixed_candidates, grid_stride_blocks(n), kThreads, 0, s, n, plan.keep_col.p, plan.l.p, plan.u.p,
             plan.c.p, p.bound_tol, fixed.p, fval.p, contrib.p, radius.p, st.d + 1);
  if (st.read(2)[1] == 0) return;
  row_gather_shift(lp.A, lp.AT, plan.keep_row.p, fixed.p, fval.p, radius.p, row_err.p, s);
  GPP_LAUNCH(fixed_filter, grid_stride_blocks(n), kThreads, 0, s, n, lp.AT.ptr, lp.AT.idx, plan.keep_row.p,
             plan.l.p, plan.u.p, row_err.p, 0.1 * p.feasibility_tol, fixed.p, contrib.p, st.d);
  if (st.read(1)[0] == 0) return;
  row_gather_shift(lp.A, lp.AT, plan.keep_row.p, fixed.p, fval.p, nullptr, shift.p, s);
  GPP_LAUNCH(fixed_apply, grid_stride_blocks(std::max(n, m)), kThreads, 0, s, n, m, fixed.p, fval.p, shift.p,
             plan.keep_col.p, plan.l.p, plan.u.p, plan.AL.p, plan.AU.p);
  plan.obj_delta += domain_objective(contrib.p, plan.rule_entry_keep_col, n, s);
  plan.has_col_action = plan.has_change = true;
}

void rule_empty_columns(Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int n = lp.n();
  if (n == 0) return;
  auto s = ctx().stream;
  DBuf<uint8_t> fixed(size_t(n), s);
  DBuf<double> fval(size_t(n), s), contrib(size_t(n), s);
  Status st;
  st.clear(3);
  GPP_LAUNCH(empty_columns_classify, grid_stride_blocks(n), kThreads, 0, s, n, plan.keep_col.p, stats.empty_col.p,
             plan.c.p, plan.l.p, plan.u.p, p.bound_tol, p.zero_tol, fixed.p, fval.p, contrib.p, st.d);
  const int32_t* f = st.read(3);
  if (f[0]) { plan.has_infeasible = true; return; }
  if (f[1]) { plan.has_unbounded = true; return; }
  if (!f[2]) return;
  GPP_LAUNCH(fix_columns, grid_stride_blocks(n), kThreads, 0, s, n, fixed.p, fval.p, plan.keep_col.p, plan.l.p,
             plan.u.p);
  plan.obj_delta += domain_objective(contrib.p, plan.rule_entry_keep_col, n, s);
  plan.has_col_action = plan.has_change = true;
}

void rule_empty_rows(Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m();
  if (m == 0) return;
  auto s = ctx().stream;
  Status st;
  st.clear(2);
  GPP_LAUNCH(empty_rows_kernel, grid_stride_blocks(m), kThreads, 0, s, m, plan.keep_row.p, stats.row_nnz.p,
             plan.AL.p, plan.AU.p, p.feasibility_tol, st.d, 0);
  const int32_t* f = st.read(2);
  if (f[0]) { plan.has_infeasible = true; return; }
  if (!f[1]) return;
  GPP_LAUNCH(empty_rows_kernel, grid_stride_blocks(m), kThreads, 0, s, m, plan.keep_row.p, stats.row_nnz.p,
             plan.AL.p, plan.AU.p, p.feasibility_tol, st.d, 1);
  plan.has_row_action = plan.has_row_deletion = plan.has_change = true;
}

void rule_singleton_rows(Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (m == 0) return;
  auto s = ctx().stream;
  DBuf<double> cl(size_t(n), s), cu(size_t(n), s);
  DBuf<uint8_t> remove(size_t(m), s);
  cl.copy_from(plan.l.p, size_t(n));
  cu.copy_from(plan.u.p, size_t(n));
  Status st;
  st.clear(3);
  GPP_LAUNCH(singleton_row_bounds, grid_stride_blocks(m), kThreads, 0, s, m, n, plan.keep_row.p,
             stats.singleton_row.p, stats.srow_col.p, stats.srow_val.p, plan.AL.p, plan.AU.p, p.zero_tol, cl.p,
             cu.p, remove.p);
  GPP_LAUNCH(singleton_rows_check, grid_stride_blocks(std::max(m, n)), kThreads, 0, s, m, n, cl.p, cu.p, plan.l.p,
             plan.u.p, remove.p, p.bound_tol, st.d);
  const int32_t* f = st.read(3);
  if (f[0]) { plan.has_infeasible = true; return; }
  if (!f[1] && !f[2]) return;
  const bool removed = f[1] != 0;
  GPP_LAUNCH(singleton_rows_commit, grid_stride_blocks(m), kThreads, 0, s, m, n, remove.p, plan.keep_row.p);
  std::swap(plan.l, cl);
  std::swap(plan.u, cu);
  plan.has_row_action = plan.has_change = true;
  plan.has_row_deletion = plan.has_row_deletion || removed;
}

}  // namespace gpp
