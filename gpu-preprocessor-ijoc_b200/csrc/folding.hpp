// Symmetry folding (colour refinement + quotient LP) and unfolding.
// Reference: cpp/src/folding/ (folding.cu:69-133, folding_refinement.cu,
// folding_reduce.cu, folding_map.cu).
#pragma once

#include "engine.cuh"

namespace gpp {

struct FoldingResult {
  bool applied = false;
  gpp_lp folded{};            // device arrays owned by this result when applied
  int32_t original_rows = 0, original_cols = 0, folded_rows = 0, folded_cols = 0;
  DBuf<int32_t> row_color, col_color;
  DBuf<double> row_scale, col_scale;
  double seconds = 0.0;
};

// run_folding (folding.cu:69-133).  Leaves `out.applied` false when the
// refinement finds no symmetry worth folding.
void run_folding(const gpp_lp& lp, double tolerance, FoldingResult& out);
void free_folding(FoldingResult& f);
// unfold_solution_device_to_host (folding_map.cu:318-380).
void unfold_to_host(const FoldingResult& f, const double* x, const double* y, const double* z, double* x_out,
                    double* y_out, double* z_out);

// Parallel-row hashes (rule_parallel_rows.cu:132-343).
void parallel_row_hashes(const DevCsr& A, const uint8_t* keep_row, const uint8_t* keep_col, int mode,
                         uint64_t* hashes, cudaStream_t s);

}  // namespace gpp
