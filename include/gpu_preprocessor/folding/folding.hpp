// Folding and pipeline entry points of the C++ layer (GPU-Preprocessor's
// cpp/include/gpu_preprocessor/folding/folding.hpp:10-58), over
// gpp_preprocess / gpp_run_presolve / gpp_postprocess / gpp_export_folding_map
// / gpp_unfold_solution.
#pragma once

#include <cstdint>
#include <vector>

#include "gpu_preprocessor/detail/status.hpp"
#include "gpu_preprocessor/folding/folding_structs.hpp"

namespace gpu_preprocessor::folding {

namespace detail {
inline FoldingPipelineSummary pipeline_view(const gpp_summary& s, double input_obj_constant) {
  FoldingPipelineSummary p;
  p.preprocessing_seconds = s.preprocessing_seconds;
  p.presolve_enabled = s.presolve_enabled != 0;
  p.folding_applied = s.folding_applied != 0;
  p.original_rows = s.original_rows;
  p.original_cols = s.original_cols;
  p.folded_rows = s.folded_rows;
  p.folded_cols = s.folded_cols;
  p.folding.applied = p.folding_applied;
  p.folding.original_rows = s.original_rows;
  p.folding.original_cols = s.original_cols;
  p.folding.folded_rows = s.folded_rows;
  p.folding.folded_cols = s.folded_cols;
  p.folding.map.original_rows = s.original_rows;
  p.folding.map.original_cols = s.original_cols;
  p.folding.map.reduced_rows = s.folded_rows;
  p.folding.map.reduced_cols = s.folded_cols;
  p.presolve = presolve::detail::presolve_view(s, input_obj_constant);
  p.folding.map.owner = p.folding_applied ? &p.presolve.record.handle : nullptr;
  return p;
}
}  // namespace detail

// The first value of every colour: a warm start of the folded model taken
// from one of the original model.  Colours are 1-based.
inline std::vector<double> fold_initial_vector(const std::vector<double>* value,
                                               const std::vector<std::int32_t>& color_index,
                                               std::int32_t reduced_length) {
  if (value == nullptr) return {};
  std::vector<double> folded(static_cast<std::size_t>(reduced_length), 0.0);
  std::vector<char> taken(static_cast<std::size_t>(reduced_length), 0);
  for (std::size_t k = 0; k < color_index.size(); ++k) {
    const auto c = static_cast<std::size_t>(color_index[k] - 1);
    if (!taken[c]) {
      folded[c] = (*value)[k];
      taken[c] = 1;
    }
  }
  return folded;
}

inline FoldingMapHost copy_map_to_host(const FoldingMapDevice& map) {
  FoldingMapHost h;
  h.original_rows = map.original_rows;
  h.original_cols = map.original_cols;
  h.reduced_rows = map.reduced_rows;
  h.reduced_cols = map.reduced_cols;
  if (map.owner == nullptr && map.run.handle == nullptr) return h;
  h.row_color_id.resize(static_cast<std::size_t>(map.original_rows));
  h.col_color_id.resize(static_cast<std::size_t>(map.original_cols));
  h.row_scale.resize(static_cast<std::size_t>(map.original_rows));
  h.col_scale.resize(static_cast<std::size_t>(map.original_cols));
  gpu_preprocessor::detail::throw_on_status(
      map.owner ? gpp_export_folding_map(map.owner, h.row_color_id.data(), h.col_color_id.data(),
                                         h.row_scale.data(), h.col_scale.data())
                : gpp_folding_run_export_map(&map.run, h.row_color_id.data(), h.col_color_id.data(),
                                             h.row_scale.data(), h.col_scale.data()),
      "copy_map_to_host");
  return h;
}

// run_folding (folding/folding.hpp:16-18): folding alone.  When it applies,
// the folded model and the map are device arrays owned by the summary until
// free_folded_lp; otherwise the summary carries the original sizes only.
// `verbose` is accepted for source compatibility and prints nothing.
inline FoldingRunSummary run_folding(const presolve::LPInfoGpu& original_model, double tolerance,
                                     bool verbose = false) {
  (void)verbose;
  gpp_folding_run r{};
  gpu_preprocessor::detail::throw_on_status(gpp_run_folding(presolve::detail::as_c(&original_model), tolerance, &r),
                                            "run_folding");
  FoldingRunSummary s;
  s.applied = r.applied != 0;
  s.original_rows = r.original_rows;
  s.original_cols = r.original_cols;
  s.folded_rows = r.folded_rows;
  s.folded_cols = r.folded_cols;
  s.profile.total_seconds = r.seconds;
  s.map.original_rows = r.original_rows;
  s.map.original_cols = r.original_cols;
  s.map.reduced_rows = r.folded_rows;
  s.map.reduced_cols = r.folded_cols;
  if (s.applied) {
    s.map.row_color_id = r.row_color_id;
    s.map.col_color_id = r.col_color_id;
    s.map.row_scale = r.row_scale;
    s.map.col_scale = r.col_scale;
    s.map.owns_buffers = true;
    s.map.run = r;
    s.folded_lp = presolve::detail::from_c(r.folded_lp);
    s.owns_folded_lp = true;
  }
  return s;
}

// free_folded_lp (folding/folding.hpp:20): releases the folded model and the
// map of a run_folding summary; safe to call twice.
inline void free_folded_lp(FoldingRunSummary& summary) {
  gpp_free_folding_run(&summary.map.run);
  summary.map.row_color_id = summary.map.col_color_id = nullptr;
  summary.map.row_scale = summary.map.col_scale = nullptr;
  summary.map.owns_buffers = false;
  summary.folded_lp = presolve::LPInfoGpu{};
  summary.owns_folded_lp = false;
}

// x_j = x_f[C(j)], z_j = z_f[C(j)] / |C(j)|, y_i = y_f[R(i)] / |R(i)|.
inline void unfold_solution(const FoldingMapHost& map, const std::vector<double>& x_red,
                            const std::vector<double>& y_red, const std::vector<double>& z_red,
                            std::vector<double>* x, std::vector<double>* y, std::vector<double>* z) {
  x->assign(static_cast<std::size_t>(map.original_cols), 0.0);
  y->assign(static_cast<std::size_t>(map.original_rows), 0.0);
  z->assign(static_cast<std::size_t>(map.original_cols), 0.0);
  for (std::size_t j = 0; j < x->size(); ++j) {
    const auto c = static_cast<std::size_t>(map.col_color_id[j] - 1);
    (*x)[j] = x_red[c];
    (*z)[j] = z_red[c] * map.col_scale[j];
  }
  for (std::size_t i = 0; i < y->size(); ++i)
    (*y)[i] = y_red[static_cast<std::size_t>(map.row_color_id[i] - 1)] * map.row_scale[i];
}

inline UnfoldedSolutionHost unfold_solution_to_host(const FoldingMapDevice& map, const std::vector<double>& x_red,
                                                    const std::vector<double>& y_red,
                                                    const std::vector<double>& z_red) {
  UnfoldedSolutionHost out;
  unfold_solution(copy_map_to_host(map), x_red, y_red, z_red, &out.x, &out.y, &out.z);
  return out;
}

// Device folded solution -> host original solution; a null input leaves the
// matching output empty.
inline UnfoldedSolutionHost unfold_solution_device_to_host(const FoldingMapDevice& map, const double* x_red,
                                                           const double* y_red, const double* z_red) {
  UnfoldedSolutionHost out;
  if (x_red) out.x.resize(static_cast<std::size_t>(map.original_cols));
  if (y_red) out.y.resize(static_cast<std::size_t>(map.original_rows));
  if (z_red) out.z.resize(static_cast<std::size_t>(map.original_cols));
  if (map.owner == nullptr && map.run.handle == nullptr)
    throw std::invalid_argument("unfold_solution_device_to_host: folding did not apply");
  double* xo = x_red ? out.x.data() : nullptr;
  double* yo = y_red ? out.y.data() : nullptr;
  double* zo = z_red ? out.z.data() : nullptr;
  gpu_preprocessor::detail::throw_on_status(
      map.owner ? gpp_unfold_solution(map.owner, x_red, y_red, z_red, xo, yo, zo)
                : gpp_folding_run_unfold(&map.run, x_red, y_red, z_red, xo, yo, zo),
      "unfold_solution_device_to_host");
  return out;
}

// Presolve alone (no folding); with params.enable_presolve false the record is
// the identity and the reduced LP borrows the input.
inline presolve::GpuPresolveSummary run_optional_gpu_presolve(const presolve::LPInfoGpu& lp,
                                                              const presolve::PresolveParams& params,
                                                              bool keep_reduced_lp) {
  return presolve::detail::run_presolve(lp, params, keep_reduced_lp);
}

// Folding (when params.enable_folding) then presolve (when
// params.enable_presolve).  The engine keeps the reduced model and the folding
// map until free_summary whatever the two keep flags say.
inline FoldingPipelineSummary run_gpu_presolve_with_folding(const presolve::LPInfoGpu& lp,
                                                            const presolve::PresolveParams& params,
                                                            bool keep_reduced_lp, bool keep_folded_lp) {
  (void)keep_reduced_lp;
  (void)keep_folded_lp;
  const gpp_params c = presolve::detail::to_c(params);
  gpp_summary s{};
  gpu_preprocessor::detail::throw_on_status(gpp_preprocess(presolve::detail::as_c(&lp), &c, &s),
                                            "run_gpu_presolve_with_folding");
  return detail::pipeline_view(s, lp.obj_constant);
}

// Reduced device solution -> original host solution (postsolve, then unfold
// when folding applied).  A null input leaves the matching output zero.
inline UnfoldedSolutionHost postsolve_and_unfold_to_host(double* x_red, double* y_red, double* z_red,
                                                         const FoldingPipelineSummary& summary,
                                                         const presolve::LPInfoGpu* original_model = nullptr) {
  UnfoldedSolutionHost out;
  out.x.assign(static_cast<std::size_t>(summary.original_cols), 0.0);
  out.y.assign(static_cast<std::size_t>(summary.original_rows), 0.0);
  out.z.assign(static_cast<std::size_t>(summary.original_cols), 0.0);
  gpu_preprocessor::detail::throw_on_status(
      gpp_postprocess(x_red, y_red, z_red, &summary.presolve.record.handle, presolve::detail::as_c(original_model),
                      out.x.data(), out.y.data(), out.z.data()),
      "postsolve_and_unfold_to_host");
  return out;
}

}  // namespace gpu_preprocessor::folding
