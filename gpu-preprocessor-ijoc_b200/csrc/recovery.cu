// GPU-resident recovery record: original-index maps, fixed-value segments and
// the chronological postsolve tape.
//
// Reference: cpp/src/presolve/device_recovery.cu:42-276,881-1027.  Rules
// write records with the indices of the current (physical) model; capture
// rewrites them to original indices with the current maps, so the tape that
// postsolve replays is expressed in the original model throughout.
#include "engine.cuh"

namespace gpp {

namespace {

__global__ void iota(int32_t* a, int32_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    a[i] = int32_t(i);
}

__device__ __forceinline__ int map_idx(int x, const int32_t* map, int n) { return x >= 0 && x < n ? map[x] : x; }

// Record types (the reference's PostsolveReductionType numbering).
enum : int {
  kFixedVariable = 0, kInfiniteBoundDualFix = 1, kSingletonColumnSubstitution = 2, kParallelColumn = 3,
  kParallelRow = 4, kDeletedRow = 5, kRowLowerBoundChange = 8, kRowUpperBoundChange = 9, kRowDualShift = 10,
  kVariableBoundChange = 11, kRowImpliedBoundChange = 12, kDoubletonEquation = 13, kFmeCol = 14
};

// One thread per record; long supports are walked by the same thread (the
// records with long index lists are rare and bounded by the row length).
__global__ void globalize_kernel(int64_t count, const int32_t* __restrict__ types, const int64_t* __restrict__ is,
                                 int32_t* __restrict__ idx, const int32_t* __restrict__ rows, int m,
                                 const int32_t* __restrict__ cols, int n) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < count; k += int64_t(gridDim.x) * blockDim.x) {
    int32_t* id = idx + is[k];
    const int64_t sz = is[k + 1] - is[k];
    switch (types[k]) {
      case kFixedVariable:
        if (sz) { id[0] = map_idx(id[0], cols, n); for (int64_t q = 1; q < sz; ++q) id[q] = map_idx(id[q], rows, m); }
        break;
      case kInfiniteBoundDualFix:
        if (sz >= 3) {
          id[1] = map_idx(id[1], cols, n);
          int64_t q = 3;
          while (q < sz) {
            const int len = id[q++];
            for (int r = 0; r < len && q < sz; ++r, ++q) id[q] = map_idx(id[q], cols, n);
          }
        }
        break;
      case kSingletonColumnSubstitution:
        if (sz >= 3) {
          id[0] = map_idx(id[0], cols, n);
          id[1] = map_idx(id[1], rows, m);
          for (int r = 0; r < id[2] && 3 + r < sz; ++r) id[3 + r] = map_idx(id[3 + r], cols, n);
        }
        break;
      case kParallelColumn:
        if (sz >= 2) { id[0] = map_idx(id[0], cols, n); id[1] = map_idx(id[1], cols, n); }
        break;
      case kParallelRow:
        if (sz >= 2) { id[0] = map_idx(id[0], rows, m); id[1] = map_idx(id[1], rows, m); }
        break;
      case kDeletedRow:
        if (sz) { id[0] = map_idx(id[0], rows, m); if (sz >= 2) id[1] = map_idx(id[1], cols, n); }
        break;
      case kRowLowerBoundChange: case kRowUpperBoundChange: case kRowDualShift:
        if (sz) id[0] = map_idx(id[0], rows, m);
        break;
      case kVariableBoundChange:
        if (sz) id[0] = map_idx(id[0], cols, n);
        break;
      case kRowImpliedBoundChange:
        if (sz >= 2) { id[0] = map_idx(id[0], cols, n); id[1] = map_idx(id[1], rows, m); }
        break;
      case kDoubletonEquation:
        if (sz >= 4) {
          id[0] = map_idx(id[0], cols, n);
          id[1] = map_idx(id[1], cols, n);
          id[2] = map_idx(id[2], rows, m);
          for (int r = 0; r < id[3] && 4 + r < sz; ++r) id[4 + r] = map_idx(id[4 + r], rows, m);
        }
        break;
      case kFmeCol:
        // [K, col, rows[K], terms, L, (orient, len)[L], cols[terms]].
        if (sz >= 4) {
          const int k_rows = id[0];
          id[1] = map_idx(id[1], cols, n);
          for (int r = 0; r < k_rows && 2 + r < sz; ++r) id[2 + r] = map_idx(id[2 + r], rows, m);
          if (3 + k_rows < sz) {
            const int terms = id[2 + k_rows], exprs = id[3 + k_rows];
            const int64_t first = int64_t(4 + k_rows) + 2 * int64_t(exprs);
            for (int t = 0; t < terms && first + t < sz; ++t) id[first + t] = map_idx(id[first + t], cols, n);
          }
        }
        break;
      default:
        break;
    }
  }
}

__global__ void fixed_flags(int32_t n, const uint8_t* __restrict__ keep, const uint8_t* __restrict__ prior,
                            const double* __restrict__ l, const double* __restrict__ u, int32_t* __restrict__ flag) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    flag[i] = (!prior || prior[i]) && !keep[i] && isfinite(l[i]) && isfinite(u[i]) && fabs(l[i] - u[i]) <= 1e-9;
}
__global__ void fixed_pack(int32_t n, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                           const double* __restrict__ l, const double* __restrict__ u, const int32_t* __restrict__ cols,
                           int32_t* __restrict__ out_idx, double* __restrict__ out_val) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    if (flag[i]) {
      out_idx[pos[i]] = cols[i];
      out_val[pos[i]] = 0.5 * (l[i] + u[i]);
    }
}

__global__ void globalize_ids(int32_t* __restrict__ ids, int64_t n, const int32_t* __restrict__ cols) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    ids[i] = cols[ids[i]];
}

}  // namespace

void capture_absolute_value(Record& r, AbsValueRecovery&& step) {
  // update_device_recovery (device_recovery.cu:912-928): column ids through
  // the record's current map, a checkpoint at the current tape length.
  auto s = ctx().stream;
  auto glob = [&](DBuf<int32_t>& ids, int64_t n) {
    GPP_LAUNCH(globalize_ids, grid_stride_blocks(n), kThreads, 0, s, ids.p, n, r.cols.p);
  };
  glob(step.split_t, step.splits);
  glob(step.split_e, step.splits);
  glob(step.pair_bound, step.pairs);
  glob(step.pair_free, step.pairs);
  glob(step.link_slack, step.links);
  glob(step.link_t, step.links);
  glob(step.max_slack, step.max_groups);
  glob(step.max_t, step.max_entries);
  r.timeline.push_back(RecoveryCheckpoint{0, int32_t(r.absval.size()), r.records});
  r.absval.push_back(std::move(step));
}

void capture_variable_pair(Record& r, VarPairRecovery&& step) {
  // update_device_recovery (device_recovery.cu:929-941).
  auto s = ctx().stream;
  for (DBuf<int32_t>* ids : {&step.plus, &step.minus, &step.root_plus, &step.root_minus})
    GPP_LAUNCH(globalize_ids, grid_stride_blocks(step.count), kThreads, 0, s, ids->p, step.count, r.cols.p);
  r.timeline.push_back(RecoveryCheckpoint{1, int32_t(r.varpair.size()), r.records});
  r.varpair.push_back(std::move(step));
}

void init_record(Record& r, int32_t m, int32_t n) {
  auto s = ctx().stream;
  r.m0 = r.m = m;
  r.n0 = r.n = n;
  r.rows.alloc(size_t(m), s);
  r.cols.alloc(size_t(n), s);
  GPP_LAUNCH(iota, grid_stride_blocks(m), kThreads, 0, s, r.rows.p, m);
  GPP_LAUNCH(iota, grid_stride_blocks(n), kThreads, 0, s, r.cols.p, n);
}

PostsolveSegment make_segment(int64_t count, int64_t n_idx, int64_t n_val) {
  auto s = ctx().stream;
  PostsolveSegment seg;
  seg.count = count;
  seg.n_idx = n_idx;
  seg.n_val = n_val;
  seg.types.alloc(size_t(count), s);
  seg.is.alloc(size_t(count) + 1, s);
  seg.vs.alloc(size_t(count) + 1, s);
  seg.idx.alloc(size_t(n_idx), s);
  seg.val.alloc(size_t(n_val), s);
  return seg;
}

void globalize_segment(PostsolveSegment& seg, const Record& r, cudaStream_t st) {
  GPP_LAUNCH(globalize_kernel, grid_stride_blocks(seg.count), kThreads, 0, st, seg.count, seg.types.p, seg.is.p,
             seg.idx.p, r.rows.p, r.m, r.cols.p, r.n);
}

void capture_tape(Record& r, std::vector<PostsolveSegment>& tape) {
  for (auto& seg : tape) {
    if (!seg.count) continue;
    globalize_segment(seg, r, ctx().stream);
    r.records += seg.count;
    r.indices += seg.n_idx;
    r.values += seg.n_val;
    r.segments.push_back(std::move(seg));
  }
  tape.clear();
}

void append_fixed(Record& r, const uint8_t* keep_col, const uint8_t* prior, const double* l, const double* u,
                  int32_t n) {
  // append_fixed (device_recovery.cu:233-276).
  if (!n) return;
  auto s = ctx().stream;
  DBuf<int32_t> flag(size_t(n) + 1, s), pos(size_t(n) + 1, s);
  GPP_LAUNCH(fixed_flags, grid_stride_blocks(n), kThreads, 0, s, n, keep_col, prior, l, u, flag.p);
  exclusive_scan_i32(flag.p, pos.p, n, s);
  const int32_t count = read_scalar(pos.p + n);
  if (!count) return;
  FixedSegment f;
  f.count = count;
  f.idx.alloc(size_t(count), s);
  f.val.alloc(size_t(count), s);
  GPP_LAUNCH(fixed_pack, grid_stride_blocks(n), kThreads, 0, s, n, flag.p, pos.p, l, u, r.cols.p, f.idx.p, f.val.p);
  r.fixed.push_back(std::move(f));
}

}  // namespace gpp
