// Bound strengthening: one Jacobi round of activity-based implied column
// bounds, finalisation (margins, near-fixing, free-zero-cost guard), support
// rows for the postsolve tape, and the fixed-column row shift.
//
// Reference: rules/rule_bound_strengthening.cu:336-813 (kernels) and
// :1176-1557 (driver).  Candidate bounds are combined with CAS max/min, whose
// result does not depend on the order of the updates.
#include <climits>

#include "engine.cuh"

namespace gpp {

namespace {


struct RowSummary {
  const double* mn;
  const double* mx;
  const int32_t* ni;
  const int32_t* pi;
};

// Implied bounds of the column of entry a from its row (reference :349-430).
__device__ __forceinline__ void implied_bounds(double a, double lj, double uj, double al, double au, double mn,
                                               double mx, int ni, int pi, double& il, double& iu) {
  double tmin, tmax;
  if (a >= 0.0) { tmin = a * lj; tmax = a * uj; } else { tmin = a * uj; tmax = a * lj; }
  double rmin, rmax;
  if (isfinite(tmin)) rmin = ni == 0 ? mn - tmin : -INFINITY;
  else if (tmin < 0.0) rmin = ni > 1 ? -INFINITY : mn;
  else rmin = mn;
  if (isfinite(tmax)) rmax = pi == 0 ? mx - tmax : INFINITY;
  else if (tmax > 0.0) rmax = pi > 1 ? INFINITY : mx;
  else rmax = mx;
  il = -INFINITY;
  iu = INFINITY;
  if (a > 0.0) {
    if (isfinite(al) && isfinite(rmax)) il = (al - rmax) / a;
    if (isfinite(au) && isfinite(rmin)) iu = (au - rmin) / a;
  } else {
    if (isfinite(au) && isfinite(rmin)) il = (au - rmin) / a;
    if (isfinite(al) && isfinite(rmax)) iu = (al - rmax) / a;
  }
}

struct CandArgs {
  const offset_t* ptr;
  const int32_t* idx;
  const double* val;
  const uint8_t* keep_row;
  const int32_t* row_nnz;
  const double* AL;
  const double* AU;
  const double2* lu;   // packed column bounds, removed columns marked
  RowSummary rs;
  double zero_tol;
  double* cand_l;
  double* cand_u;
};

// The row's sides and activity summary, loaded once per row.
struct RowCtx {
  double al, au, mn, mx;
  int ni, pi;
};
__device__ __forceinline__ RowCtx row_ctx(const CandArgs& g, int i) {
  return RowCtx{g.AL[i], g.AU[i], g.rs.mn[i], g.rs.mx[i], g.rs.ni[i], g.rs.pi[i]};
}

// Candidate bounds of column j from one entry a of a row (reference
// :373-430); b holds the column's current bounds.
__device__ __forceinline__ void candidate_update(const CandArgs& g, const RowCtx& rc, int j, double a, double2 b) {
  const double ol = b.x, ou = b.y;
  double il, iu;
  implied_bounds(a, ol, ou, rc.al, rc.au, rc.mn, rc.mx, rc.ni, rc.pi, il, iu);
  double nl = ol, nu = ou;
  if (isfinite(il)) nl = fmax(nl, il);
  if (isfinite(iu)) nu = fmin(nu, iu);
  if (nl > ol) red_max_f64(&g.cand_l[j], nl);
  if (nu < ou) red_min_f64(&g.cand_u[j], nu);
}

// Entry-parallel form of the candidate sweep: the candidates are combined by
// atomic max / min, which is order-free, so instead of row roles every thread
// takes consecutive stored entries (coalesced loads, full memory-level
// parallelism) and finds their row by a binary search over the tile's row
// pointers, staged in shared memory.
constexpr int kTileRows = 2048;

__global__ void __launch_bounds__(kThreads)
candidates_entries(offset_t nnz, const int2* __restrict__ tile_rows, CandArgs g) {
  __shared__ offset_t sptr[kTileRows + 1];
  const L2Hints hint = l2_hints();
  for (offset_t base = offset_t(blockIdx.x) * kEntryTile; base < nnz; base += offset_t(gridDim.x) * kEntryTile) {
    const offset_t last = min(nnz, base + kEntryTile) - 1;
    const int2 span = tile_rows[base / kEntryTile];   // rows of the tile's first and last entry
    const int r0 = span.x, r1 = span.y;
    const bool staged = r1 - r0 + 1 <= kTileRows;
    if (staged)
      for (int k = threadIdx.x; k <= r1 - r0 + 1; k += kThreads) sptr[k] = g.ptr[r0 + k];
    __syncthreads();
    // The next entry's index and value are loaded one iteration ahead, so an
    // entry's critical path starts at its gather.
    constexpr int K = kEntryTile / kThreads;
    offset_t p = base + threadIdx.x;
    int j = p <= last ? ld_stream(g.idx + p, hint.stream) : -1;
    double a = p <= last ? ld_stream(g.val + p, hint.stream) : 0.0;
    for (int k = 0; k < K && p <= last; ++k, p += kThreads) {
      const offset_t pn = p + kThreads;
      const bool next = k + 1 < K && pn <= last;
      const int jn = next ? ld_stream(g.idx + pn, hint.stream) : -1;
      const double an = next ? ld_stream(g.val + pn, hint.stream) : 0.0;
      const int i = staged ? r0 + row_of(sptr, 0, r1 - r0 + 1, p) : row_of(g.ptr, r0, r1 + 1, p);
      // Every load of the entry at once (the column's bounds do not depend on
      // the row; the row's flags and summary come from one or two lines that
      // the warp's neighbouring entries share), so an entry waits for one
      // memory round trip instead of two.
      const double2 b = ld_keep(g.lu + j, hint.keep);
      const bool row_live = (g.keep_row[i] != 0) & (g.row_nnz[i] > 1);
      const RowCtx rc = row_ctx(g, i);
      if (row_live && !removed_column(b) && !(fabs(a) <= g.zero_tol)) candidate_update(g, rc, j, a, b);
      j = jn;
      a = an;
    }
    __syncthreads();
  }
}

// _kernel_finalize_bound_strengthening (reference :646-796).
__global__ void finalize_kernel(int n, const uint8_t* __restrict__ keep_col, const double* __restrict__ l,
                                const double* __restrict__ u, const double* __restrict__ cand_l,
                                const double* __restrict__ cand_u, const double* __restrict__ ref_l,
                                const double* __restrict__ ref_u, const double* __restrict__ c,
                                const double* __restrict__ vmax_arr, int preserve_free_zero_cost, double zero_tol,
                                double ft, double upper_relax, double* __restrict__ fl, double* __restrict__ fu,
                                uint8_t* __restrict__ lch, uint8_t* __restrict__ uch, uint8_t* __restrict__ fx,
                                double* __restrict__ fixv, int32_t* __restrict__ status) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double lj = l[j], uj = u[j];
    if (!keep_col[j]) {
      fl[j] = lj; fu[j] = uj; lch[j] = uch[j] = fx[j] = 0; fixv[j] = 0.0;
      continue;
    }
    double cl = cand_l[j], cu = cand_u[j];
    const double vmax = vmax_arr[j];
    double nl = lj, nu = uj;
    uint8_t lc = 0, uc = 0, fj = 0;
    double fat = 0.0;
    double el = lj, eu = uj;
    if (isfinite(cl)) el = fmax(el, cl);
    if (isfinite(cu)) eu = fmin(eu, cu);
    if (el > eu + ft) { atomicMax(status + 0, 1); continue; }
    const bool was_free = !isfinite(ref_l[j]) && !isfinite(ref_u[j]);
    const bool box = isfinite(cl) && isfinite(cu);
    const bool zero_cost = fabs(c[j]) <= zero_tol;
    const bool nearly_fixed = box && (cu <= cl || (cu - cl) * vmax <= ft);
    if (preserve_free_zero_cost && was_free && box && zero_cost && !nearly_fixed) { cl = lj; cu = uj; }
    if (isfinite(cl) && cl > lj && isfinite(uj)) {
      if (cl >= uj + ft) { atomicMax(status + 0, 1); continue; }
      if (cl >= uj || (uj - cl) * vmax <= ft) { fj = 1; fat = uj; nl = uj; nu = uj; }
    }
    if (!fj && isfinite(cl) && cl > lj) {
      const bool tighten = !isfinite(lj) || ((cl - lj > ft * 1.0e4) && (cl - lj > 1.0e-2 * fabs(lj)));
      if (tighten) {
        if (cl != nearbyint(cl)) cl -= 0.5 * ft * fabs(cl);
        nl = cl;
        lc = 1;
      }
    }
    if (!fj && isfinite(cu) && cu < uj && isfinite(nl)) {
      if (cu <= nl - ft) { atomicMax(status + 0, 1); continue; }
      if (cu <= nl || (cu - nl) * vmax <= ft) { fj = 1; fat = nl; nu = nl; }
    }
    if (!fj && isfinite(cu) && cu < uj) {
      const bool tighten = !isfinite(uj) || ((uj - cu > ft * 1.0e4) && (uj - cu > 1.0e-2 * fabs(uj)));
      if (tighten) {
        if (cu != nearbyint(cu)) cu += upper_relax * ft * fabs(cu);
        nu = cu;
        uc = 1;
      }
    }
    if (fj) { lc = uc = 0; atomicMax(status + 2, 1); }
    if (lc || uc) atomicMax(status + 1, 1);
    fl[j] = nl; fu[j] = nu; lch[j] = lc; uch[j] = uc; fx[j] = fj; fixv[j] = fat;
  }
}

// Support rows and per-column tape sizes (reference :815-960, :970-1008).
__global__ void support_kernel(int n, const offset_t* __restrict__ at_ptr, const int32_t* __restrict__ at_idx,
                               const double* __restrict__ at_val, const uint8_t* __restrict__ keep_row,
                               const int32_t* __restrict__ row_nnz, const double* __restrict__ AL,
                               const double* __restrict__ AU, const double* __restrict__ l,
                               const double* __restrict__ u, RowSummary rs, const uint8_t* __restrict__ lch,
                               const uint8_t* __restrict__ uch, const double* __restrict__ fl,
                               const double* __restrict__ fu, double zero_tol, double tol, double support_tol,
                               int32_t* __restrict__ sup_l, int32_t* __restrict__ sup_u,
                               int64_t* __restrict__ rec_count, int64_t* __restrict__ idx_count) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    int sl = INT_MAX, su = INT_MAX;
    const bool nl = lch[j], nu = uch[j];
    if (nl || nu) {
      const double lj = l[j], uj = u[j], flj = fl[j], fuj = fu[j];
      const bool want_l = nl && flj > lj + tol, want_u = nu && fuj < uj - tol;
      // Four entries per round with every load issued before the first use
      // (one memory round trip per four entries); the support row is the
      // smallest qualifying row, which does not depend on the visiting order.
      constexpr int kBatch = 4;
      const offset_t end = at_ptr[j + 1];
      for (offset_t p0 = at_ptr[j]; p0 < end && (want_l || want_u); p0 += kBatch) {
        int row[kBatch];
        double a[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
          row[k] = p0 + k < end ? at_idx[p0 + k] : -1;
          a[k] = p0 + k < end ? at_val[p0 + k] : 0.0;
        }
        bool live[kBatch];
        double al[kBatch], au[kBatch], mn[kBatch], mx[kBatch];
        int ni[kBatch], pi[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
          const int i = row[k] >= 0 ? row[k] : 0;
          live[k] = row[k] >= 0 && (keep_row[i] != 0) & (row_nnz[i] > 1);
          al[k] = AL[i]; au[k] = AU[i]; mn[k] = rs.mn[i]; mx[k] = rs.mx[i]; ni[k] = rs.ni[i]; pi[k] = rs.pi[i];
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
          if (!live[k] || fabs(a[k]) <= zero_tol) continue;
          double il, iu;
          implied_bounds(a[k], lj, uj, al[k], au[k], mn[k], mx[k], ni[k], pi[k], il, iu);
          if (want_l && isfinite(il) && fabs(il - flj) <= support_tol) sl = min(sl, row[k]);
          if (want_u && isfinite(iu) && fabs(iu - fuj) <= support_tol) su = min(su, row[k]);
        }
      }
    }
    sup_l[j] = sl;
    sup_u[j] = su;
    rec_count[j] = int64_t(nl) + int64_t(nu);
    idx_count[j] = (nl ? (sl == INT_MAX ? 1 : 2) : 0) + (nu ? (su == INT_MAX ? 1 : 2) : 0);
  }
}

constexpr int kVariableBoundChange = 11, kRowImpliedBoundChange = 12, kFixedVariable = 0;

__global__ void pack_bound_records(int n, const uint8_t* __restrict__ lch, const uint8_t* __restrict__ uch,
                                   const int32_t* __restrict__ sup_l, const int32_t* __restrict__ sup_u,
                                   const double* __restrict__ l, const double* __restrict__ u,
                                   const double* __restrict__ fl, const double* __restrict__ fu,
                                   const int64_t* __restrict__ rec_pos, const int64_t* __restrict__ idx_pos,
                                   int32_t* __restrict__ types, int64_t* __restrict__ is, int64_t* __restrict__ vs,
                                   int32_t* __restrict__ idx, double* __restrict__ val) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (j == 0) { is[0] = 0; vs[0] = 0; }
    if (!lch[j] && !uch[j]) continue;
    int64_t k = rec_pos[j], ip = idx_pos[j];
    double cur_l = l[j];
    const double cur_u = u[j];
    auto emit = [&](int sup, double a, double b, double c2, double d) {
      types[k] = sup == INT_MAX ? kVariableBoundChange : kRowImpliedBoundChange;
      idx[ip++] = j;
      if (sup != INT_MAX) idx[ip++] = sup;
      val[4 * k] = a; val[4 * k + 1] = b; val[4 * k + 2] = c2; val[4 * k + 3] = d;
      is[k + 1] = ip;
      vs[k + 1] = 4 * (k + 1);
      ++k;
    };
    if (lch[j]) {
      emit(sup_l[j], cur_l, cur_u, fl[j], cur_u);
      cur_l = fl[j];
    }
    if (uch[j]) emit(sup_u[j], cur_l, cur_u, cur_l, fu[j]);
  }
}

__global__ void apply_bounds(int n, const double* __restrict__ fl, const double* __restrict__ fu,
                             const uint8_t* __restrict__ fx, double* __restrict__ l, double* __restrict__ u,
                             uint8_t* __restrict__ keep_col) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    l[j] = fl[j];
    u[j] = fu[j];
    if (fx[j]) keep_col[j] = 0;
  }
}

// Row shift of the fixed columns, then removal of rows left without a live
// column (feasible sides) or the infeasibility flag (reference :1083-1156).
__global__ void shift_and_empty_rows(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                     const double* __restrict__ shift, const uint8_t* __restrict__ keep_col,
                                     uint8_t* __restrict__ keep_row, double* __restrict__ AL,
                                     double* __restrict__ AU, double ft, int32_t* __restrict__ status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    AL[i] -= shift[i];
    AU[i] -= shift[i];
    if (!keep_row[i]) continue;
    int cnt = 0;
    for (offset_t p = ptr[i]; p < ptr[i + 1] && cnt == 0; ++p) cnt += keep_col[idx[p]] != 0;
    if (cnt) continue;
    if (AL[i] <= ft && AU[i] >= -ft) { keep_row[i] = 0; atomicMax(status + 4, 1); }
    else atomicMax(status + 3, 1);
  }
}

// FixedVariable records of fixed columns: (col, kept rows...), (value, c, coefficients...).
__global__ void fixed_record_sizes(int n, const uint8_t* __restrict__ fx, const offset_t* __restrict__ at_ptr,
                                   const int32_t* __restrict__ at_idx, const uint8_t* __restrict__ keep_row,
                                   int64_t* __restrict__ recs, int64_t* __restrict__ nz) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    int64_t c = 0;
    if (fx[j])
      for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p) c += keep_row[at_idx[p]] != 0;
    recs[j] = fx[j] ? 1 : 0;
    nz[j] = c;
  }
}
__global__ void fixed_record_pack(int n, const uint8_t* __restrict__ fx, const offset_t* __restrict__ at_ptr,
                                  const int32_t* __restrict__ at_idx, const double* __restrict__ at_val,
                                  const uint8_t* __restrict__ keep_row, const double* __restrict__ fixv,
                                  const double* __restrict__ c, const int64_t* __restrict__ rec_pos,
                                  const int64_t* __restrict__ nz_pos, int32_t* __restrict__ types,
                                  int64_t* __restrict__ is, int64_t* __restrict__ vs, int32_t* __restrict__ idx,
                                  double* __restrict__ val, double* __restrict__ obj_c, double* __restrict__ obj_v) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (j == 0) { is[0] = 0; vs[0] = 0; }
    if (!fx[j]) continue;
    const int64_t k = rec_pos[j], base = nz_pos[j];
    int64_t ip = k + base, vp = 2 * k + base;
    types[k] = kFixedVariable;
    idx[ip++] = j;
    val[vp++] = fixv[j];
    val[vp++] = c[j];
    for (offset_t p = at_ptr[j]; p < at_ptr[j + 1]; ++p)
      if (keep_row[at_idx[p]]) { idx[ip++] = at_idx[p]; val[vp++] = at_val[p]; }
    is[k + 1] = ip;
    vs[k + 1] = vp;
    obj_c[k] = c[j];
    obj_v[k] = fixv[j];
  }
}

// Live rows binned by infinite-term count of their minimum and maximum
// activity (0, 1, 2, >= 3): the learned schedule's histogram features.
__global__ void inf_histogram(int m, const uint8_t* __restrict__ keep_row, const int32_t* __restrict__ ni,
                              const int32_t* __restrict__ pi, uint32_t* __restrict__ hist) {
  __shared__ uint32_t bins[8];
  if (threadIdx.x < 8) bins[threadIdx.x] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    if (!keep_row[i]) continue;
    atomicAdd(&bins[min(ni[i], 3)], 1u);
    atomicAdd(&bins[4 + min(pi[i], 3)], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 8 && bins[threadIdx.x]) atomicAdd(hist + threadIdx.x, bins[threadIdx.x]);
}

}  // namespace

void rule_bound_strengthening(Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  if (m == 0 || n == 0) return;
  auto s = ctx().stream;
  DBuf<double> cl(size_t(n), s), cu(size_t(n), s), mn(size_t(m), s), mx(size_t(m), s), vmax(size_t(n), s);
  DBuf<int32_t> ni(size_t(m), s), pi(size_t(m), s);
  cl.copy_from(plan.l.p, size_t(n));
  cu.copy_from(plan.u.p, size_t(n));
  Status st;
  st.clear(5);
  // One packed bounds array serves the activity sweep and the candidate sweep.
  DBuf<double2> lu(size_t(n), s);
  pack_bounds(plan.l.p, plan.u.p, plan.keep_col.p, n, lu.p, s);
  row_activity_summary_packed(lp.A, lu.p, p.zero_tol, plan.keep_row.p, stats.row_nnz.p, mn.p, mx.p, ni.p, pi.p, s);
  const RowSummary rs{mn.p, mx.p, ni.p, pi.p};
  if (plan.inf_hist) {
    check(cudaMemsetAsync(plan.inf_hist, 0, 8 * sizeof(uint32_t), s), "inf_hist");
    GPP_LAUNCH(inf_histogram, grid_stride_blocks(m), kThreads, 0, s, m, plan.keep_row.p, ni.p, pi.p, plan.inf_hist);
  }
  {
    CandArgs g{lp.A.ptr, lp.A.idx, lp.A.val, plan.keep_row.p, stats.row_nnz.p, plan.AL.p, plan.AU.p, lu.p, rs,
               p.zero_tol, cl.p, cu.p};
    const double bytes = 4.0 * (m + 1) + 12.0 * lp.A.nnz + double(m) + 4.0 * m + 16.0 * m + 24.0 * m + 16.0 * n +
                         16.0 * n;
    const RowSchedule& sch = stored_schedule(lp.A);
    GPP_LAUNCH_BYTES(candidates_entries, bytes, int(std::max<int64_t>(1, std::min<int64_t>(sch.tiles, kNumSMs * 8))),
                     kThreads, 0, s, lp.A.nnz, sch.tile_rows.p, g);
  }
  col_max_abs(lp.AT, plan.keep_row.p, vmax.p, s);
  DBuf<double> fl(size_t(n), s), fu(size_t(n), s), fixv(size_t(n), s);
  DBuf<uint8_t> lch(size_t(n), s), uch(size_t(n), s), fx(size_t(n), s);
  const double* ref_l = plan.ref_l ? plan.ref_l : plan.l.p;
  const double* ref_u = plan.ref_u ? plan.ref_u : plan.u.p;
  GPP_LAUNCH(finalize_kernel, grid_stride_blocks(n), kThreads, 0, s, n, plan.keep_col.p, plan.l.p, plan.u.p, cl.p,
             cu.p, ref_l, ref_u, plan.c.p, vmax.p, int(p.bound_strengthening_preserve_free_zero_cost), p.zero_tol,
             p.feasibility_tol, p.bound_strengthening_upper_relaxation_factor, fl.p, fu.p, lch.p, uch.p, fx.p,
             fixv.p, st.d);
  const int32_t* f = st.read(3);
  if (f[0]) { plan.has_infeasible = true; return; }
  const bool changed = f[1] != 0, fixed = f[2] != 0;
  if (!changed && !fixed) return;
  if (p.record_postsolve_tape && changed) {
    DBuf<int32_t> sl(size_t(n), s), su(size_t(n), s);
    DBuf<int64_t> rc(size_t(n) + 1, s), ic(size_t(n) + 1, s), rpos(size_t(n) + 1, s), ipos(size_t(n) + 1, s);
    const double support_tol = std::fmax(10.0 * p.bound_tol, 1.0e-10);
    GPP_LAUNCH(support_kernel, grid_stride_blocks(n), kThreads, 0, s, n, lp.AT.ptr, lp.AT.idx, lp.AT.val,
               plan.keep_row.p, stats.row_nnz.p, plan.AL.p, plan.AU.p, plan.l.p, plan.u.p, rs, lch.p, uch.p, fl.p,
               fu.p, p.zero_tol, p.bound_tol, support_tol, sl.p, su.p, rc.p, ic.p);
    exclusive_scan_i64(rc.p, rpos.p, n, s);
    exclusive_scan_i64(ic.p, ipos.p, n, s);
    const auto [recs, nidx] = read_scalars(rpos.p + n, ipos.p + n);
    if (recs) {
      PostsolveSegment seg = make_segment(recs, nidx, 4 * recs);
      GPP_LAUNCH(pack_bound_records, grid_stride_blocks(n), kThreads, 0, s, n, lch.p, uch.p, sl.p, su.p, plan.l.p,
                 plan.u.p, fl.p, fu.p, rpos.p, ipos.p, seg.types.p, seg.is.p, seg.vs.p, seg.idx.p, seg.val.p);
      plan.tape.push_back(std::move(seg));
    }
  }
  GPP_LAUNCH(apply_bounds, grid_stride_blocks(n), kThreads, 0, s, n, fl.p, fu.p, fx.p, plan.l.p, plan.u.p,
             plan.keep_col.p);
  double obj_delta = 0.0;
  if (fixed) {
    DBuf<double> shift(size_t(m), s);
    row_gather_shift(lp.A, lp.AT, plan.keep_row.p, fx.p, fixv.p, nullptr, shift.p, s);
    GPP_LAUNCH(shift_and_empty_rows, grid_stride_blocks(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, shift.p,
               plan.keep_col.p, plan.keep_row.p, plan.AL.p, plan.AU.p, p.feasibility_tol, st.d);
    const int32_t* g = st.read(5);
    if (g[3]) { plan.has_infeasible = true; return; }
    DBuf<int64_t> rc(size_t(n) + 1, s), nz(size_t(n) + 1, s), rpos(size_t(n) + 1, s), npos(size_t(n) + 1, s);
    GPP_LAUNCH(fixed_record_sizes, grid_stride_blocks(n), kThreads, 0, s, n, fx.p, lp.AT.ptr, lp.AT.idx,
               plan.keep_row.p, rc.p, nz.p);
    exclusive_scan_i64(rc.p, rpos.p, n, s);
    exclusive_scan_i64(nz.p, npos.p, n, s);
    const auto [recs, nnz] = read_scalars(rpos.p + n, npos.p + n);
    PostsolveSegment seg = make_segment(recs, recs + nnz, 2 * recs + nnz);
    DBuf<double> oc(size_t(recs), s), ov(size_t(recs), s);
    GPP_LAUNCH(fixed_record_pack, grid_stride_blocks(n), kThreads, 0, s, n, fx.p, lp.AT.ptr, lp.AT.idx, lp.AT.val,
               plan.keep_row.p, fixv.p, plan.c.p, rpos.p, npos.p, seg.types.p, seg.is.p, seg.vs.p, seg.idx.p,
               seg.val.p, oc.p, ov.p);
    // append_compact_fixed_variable_tape_from_device (fixed_variable_tape.cu:286-315):
    // objective delta accumulated in long double in column order.
    const auto [hc, hv] = to_host2(oc.p, size_t(recs), ov.p, size_t(recs));
    long double acc = 0.0L;
    for (size_t k = 0; k < hc.size(); ++k) acc += (long double)hc[k] * (long double)hv[k];
    obj_delta = double(acc);
    if (p.record_postsolve_tape) plan.tape.push_back(std::move(seg));
  }
  plan.obj_delta += obj_delta;
  plan.has_row_action = plan.has_row_action || fixed;
  plan.has_col_action = plan.has_col_action || fixed;
  plan.has_change = true;
}

}  // namespace gpp
