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
#include "engine.cuh"

namespace gpp {

namespace {

enum : int32_t { kBadRow = 1, kBadColumn = 2, kBadValue = 4, kNoWitness = 8 };

// One launch checks rows (sides and a cost-1 witness), columns (box and
// cost) and every stored coefficient of A and A^T, grid-stride over the
// largest of the three ranges.
__global__ void cd_validate(int m, int n, offset_t nnz, const offset_t* __restrict__ ptr,
                            const int32_t* __restrict__ idx, const double* __restrict__ a,
                            const double* __restrict__ at, const double* __restrict__ c,
                            const double* __restrict__ AL, const double* __restrict__ AU,
                            const double* __restrict__ l, const double* __restrict__ u,
                            int32_t* __restrict__ failure) {
  int32_t bad = 0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nnz; t += stride)
    if (a[t] != 1.0 || at[t] != 1.0) bad |= kBadValue;
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += stride) {
    const double cj = c[j];
    if (l[j] != 0.0 || u[j] != 1.0 || !(isfinite(cj) && cj >= 1.0 && floor(cj) == cj)) bad |= kBadColumn;
  }
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += stride) {
    if (AL[i] != 1.0 || !(isinf(AU[i]) && AU[i] > 0.0)) bad |= kBadRow;
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

}  // namespace

void rule_column_domination(Plan& plan, const WorkingLp& lp, const gpp_params& p) {
  if (plan.has_infeasible || plan.has_unbounded) return;
  const int m = lp.m(), n = lp.n();
  const offset_t nnz = lp.A.nnz;
  if (m <= 0 || nnz <= 0 || n < std::max(1, p.column_domination_min_fixed_cols)) return;
  auto s = ctx().stream;
  Status st;
  st.clear(2);
  GPP_LAUNCH(cd_validate, grid_stride_blocks(std::max<int64_t>(nnz, std::max(m, n))), kThreads, 0, s, m, n, nnz,
             lp.A.ptr, lp.A.idx, lp.A.val, lp.AT.val, plan.c.p, plan.AL.p, plan.AU.p, plan.l.p, plan.u.p, st.d);
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
