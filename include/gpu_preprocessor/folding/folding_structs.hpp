// Folding / pipeline structs of the C++ layer (GPU-Preprocessor's
// cpp/include/gpu_preprocessor/folding/folding_structs.hpp:59-115).
//
// The folding map stays on the device inside the summary; FoldingMapDevice is
// its sizes plus a view of the owning summary (not raw device pointers), and
// copy_map_to_host / unfold_solution_device_to_host read it through the C ABI.
// The folded model itself is internal to the engine and is not exported.
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

struct FoldingMapDevice {
  std::int32_t original_rows = 0;
  std::int32_t original_cols = 0;
  std::int32_t reduced_rows = 0;
  std::int32_t reduced_cols = 0;
  const gpp_summary* owner = nullptr;  // the summary holding the map on the device
};

struct FoldingRunSummary {
  bool applied = false;
  std::int32_t original_rows = 0;
  std::int32_t original_cols = 0;
  std::int32_t folded_rows = 0;
  std::int32_t folded_cols = 0;
  FoldingMapDevice map;
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
