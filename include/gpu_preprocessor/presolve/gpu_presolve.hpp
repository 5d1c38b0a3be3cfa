// Presolve entry points of the C++ layer (GPU-Preprocessor's
// cpp/include/gpu_preprocessor/presolve/gpu_presolve.hpp:14-40), over
// gpp_run_presolve / gpp_free_summary.
#pragma once

#include "gpu_preprocessor/detail/status.hpp"
#include "gpu_preprocessor/presolve/presolve_structs.hpp"

namespace gpu_preprocessor::presolve {

struct GpuPresolveSummary {
  std::int32_t original_rows = 0;
  std::int32_t original_cols = 0;
  std::int32_t reduced_rows = 0;
  std::int32_t reduced_cols = 0;
  NnzOffset reduced_nnz = 0;
  std::int32_t iterations = 0;
  bool stopped_at_iteration_limit = false;
  bool has_change = false;
  double elapsed_seconds = 0.0;
  double obj_constant_delta = 0.0;
  bool has_infeasible = false;
  bool has_unbounded = false;
  PresolveRecordGpu record;
  LPInfoGpu reduced_lp;
  bool owns_reduced_lp = false;
};

namespace detail {
// Presolve view of a C-ABI summary.  Presolve ran on the folded model when
// folding applied, so its "original" sizes are the folded sizes.
inline GpuPresolveSummary presolve_view(const gpp_summary& s, double input_obj_constant) {
  GpuPresolveSummary p;
  p.original_rows = s.folded_rows;
  p.original_cols = s.folded_cols;
  p.reduced_rows = s.reduced_rows;
  p.reduced_cols = s.reduced_cols;
  p.reduced_nnz = s.reduced_nnz;
  p.iterations = s.iterations;
  p.stopped_at_iteration_limit = s.stopped_at_iteration_limit != 0;
  p.has_change = s.has_change != 0;
  p.elapsed_seconds = s.elapsed_seconds;
  p.obj_constant_delta = s.obj_constant_delta;
  p.has_infeasible = s.has_infeasible != 0;
  p.has_unbounded = s.has_unbounded != 0;
  p.reduced_lp = from_c(s.reduced_lp);
  p.owns_reduced_lp = s.owns_reduced_lp != 0;
  p.record.m0 = s.folded_rows;
  p.record.n0 = s.folded_cols;
  p.record.m1 = s.reduced_rows;
  p.record.n1 = s.reduced_cols;
  p.record.obj_constant_old = input_obj_constant;
  p.record.obj_constant_new = s.reduced_lp.obj_constant;
  p.record.handle = s;
  return p;
}

inline GpuPresolveSummary run_presolve(const LPInfoGpu& lp, const PresolveParams& params, bool keep_reduced_lp) {
  const gpp_params c = to_c(params);
  gpp_summary s{};
  gpu_preprocessor::detail::throw_on_status(gpp_run_presolve(as_c(&lp), &c, keep_reduced_lp ? 1 : 0, &s),
                                            "run_gpu_presolve");
  return presolve_view(s, lp.obj_constant);
}
}  // namespace detail

// Presolve only; the reduced LP is released before return, the record kept.
inline GpuPresolveSummary run_gpu_presolve_with_record(const LPInfoGpu& lp, const PresolveParams& params) {
  return detail::run_presolve(lp, params, false);
}

// Presolve only; reduced LP and record kept until free_gpu_presolve_reduced_lp.
inline GpuPresolveSummary run_gpu_presolve_with_reduced_lp(const LPInfoGpu& lp, const PresolveParams& params) {
  return detail::run_presolve(lp, params, true);
}

// Releases the reduced LP and the record; a second call is a no-op.
inline void free_gpu_presolve_reduced_lp(GpuPresolveSummary& summary) {
  gpp_free_summary(&summary.record.handle);
  summary = GpuPresolveSummary{};
}

}  // namespace gpu_preprocessor::presolve
