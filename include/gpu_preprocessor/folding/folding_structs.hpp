// Folding / pipeline structs of the C++ layer (GPU-Preprocessor's
// cpp/include/gpu_preprocessor/folding/folding_structs.hpp:59-115).
//
// In the pipeline (run_gpu_presolve_with_folding / preprocess) the folding map
// stays on the device inside the summary, and FoldingMapDevice is its sizes
// plus a view of the owning summary.  A standalone run_folding exports what
// the reference's does: the folded model and the map as device arrays (owned
// by the run until free_folded_lp).  copy_map_to_host and
// unfold_solution_device_to_host read either kind through the C ABI.
#pragma once

#include <cstdint>
#include <vector>

#include "gpu_preprocessor/presolve/gpu_presolve.hpp"

namespace gpu_preprocessor::folding {

struct FoldingMapHost {
  std::int32_t original_rows = 0;
  std::int32_t original_cols = 0;
  std::int32_t reduced_rows = 0;
  std::int32_t reduced_cols = 0;
  std::vector<std::int32_t> row_color_id;  // 1-based colour of every original row
  std::vector<std::int32_t> col_color_id;  // 1-based colour of every original column
  std::vector<double> row_scale;           // 1 / |colour of the row|
  std::vector<double> col_scale;           // 1 / |colour of the column|
};

// Timings of a folding run.  This engine times the run as a whole
// (total_seconds); the stage fields are kept for source compatibility and
// stay zero.
struct FoldingRefinementProfile {
  double total_seconds = 0.0;
  double init_color_seconds = 0.0;
  double spmv_at_seconds = 0.0;
  double refine_col_seconds = 0.0;
  double spmv_a_seconds = 0.0;
  double refine_row_seconds = 0.0;
  std::int32_t rounds = 0;
  bool refinement_ok = false;
  std::int32_t final_row_colors = 0;
  std::int32_t final_col_colors = 0;
};

struct FoldingReduceProfile {
  double total_seconds = 0.0;
  double count_color_seconds = 0.0;
  double emit_triplet_seconds = 0.0;
  double sort_reduce_seconds = 0.0;
  double copy_unique_to_host_seconds = 0.0;
  double host_filter_rebuild_seconds = 0.0;
  double host_csr_build_seconds = 0.0;
  double copy_reduced_matrix_to_device_seconds = 0.0;
  double transpose_seconds = 0.0;
  double sum_cost_seconds = 0.0;
  double row_bounds_seconds = 0.0;
  double col_bounds_seconds = 0.0;
  NnzOffset unique_entries = 0;
  NnzOffset kept_entries = 0;
};

struct FoldingMapProfile {
  double total_seconds = 0.0;
  double copy_color_ids_seconds = 0.0;
  double count_color_seconds = 0.0;
  double scale_seconds = 0.0;
};

struct FoldingProfile {
  double total_seconds = 0.0;
  FoldingRefinementProfile refinement;
  FoldingReduceProfile reduce;
  FoldingMapProfile map;
};

struct FoldingMapDevice {
  std::int32_t original_rows = 0;
  std::int32_t original_cols = 0;
  std::int32_t reduced_rows = 0;
  std::int32_t reduced_cols = 0;
  // Device arrays of a standalone run_folding (NULL in the pipeline's view).
  std::int32_t* row_color_id = nullptr;
  std::int32_t* col_color_id = nullptr;
  double* row_scale = nullptr;
  double* col_scale = nullptr;
  bool owns_buffers = false;
  const gpp_summary* owner = nullptr;  // pipeline: the summary holding the map on the device
  gpp_folding_run run{};               // run_folding: the run holding the map
};

struct FoldingRunSummary {
  bool applied = false;
  std::int32_t original_rows = 0;
  std::int32_t original_cols = 0;
  std::int32_t folded_rows = 0;
  std::int32_t folded_cols = 0;
  FoldingProfile profile;
  FoldingMapDevice map;
  presolve::LPInfoGpu folded_lp;
  bool owns_folded_lp = false;
};

// Move-only, like the reference's (its record cannot be copied).  After a
// move, map.owner is re-pointed at this summary's own handle.
struct FoldingPipelineSummary {
  double preprocessing_seconds = 0.0;
  double workspace_setup_seconds = 0.0;
  double workspace_release_seconds = 0.0;
  bool presolve_enabled = true;
  bool folding_applied = false;
  std::int32_t original_rows = 0;
  std::int32_t original_cols = 0;
  std::int32_t folded_rows = 0;
  std::int32_t folded_cols = 0;
  FoldingRunSummary folding;
  presolve::GpuPresolveSummary presolve;

  FoldingPipelineSummary() = default;
  FoldingPipelineSummary(const FoldingPipelineSummary&) = delete;
  FoldingPipelineSummary& operator=(const FoldingPipelineSummary&) = delete;
  FoldingPipelineSummary(FoldingPipelineSummary&& o) noexcept { *this = static_cast<FoldingPipelineSummary&&>(o); }
  FoldingPipelineSummary& operator=(FoldingPipelineSummary&& o) noexcept {
    if (this != &o) {
      preprocessing_seconds = o.preprocessing_seconds;
      workspace_setup_seconds = o.workspace_setup_seconds;
      workspace_release_seconds = o.workspace_release_seconds;
      presolve_enabled = o.presolve_enabled;
      folding_applied = o.folding_applied;
      original_rows = o.original_rows;
      original_cols = o.original_cols;
      folded_rows = o.folded_rows;
      folded_cols = o.folded_cols;
      folding = o.folding;
      presolve = static_cast<presolve::GpuPresolveSummary&&>(o.presolve);
      folding.map.owner = folding.applied ? &presolve.record.handle : nullptr;
      o.folding.map.owner = nullptr;
    }
    return *this;
  }
};

struct UnfoldedSolutionHost {
  std::vector<double> x;
  std::vector<double> y;
  std::vector<double> z;
};

}  // namespace gpu_preprocessor::folding
