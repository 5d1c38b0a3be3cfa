// Engine entry points used by the C ABI layer.
#pragma once

#include <string>
#include <vector>

#include "engine.cuh"

namespace gpp {

// Everything one presolve call produces; held by the gpp_record handle.
struct PresolveOutput {
  int32_t original_rows = 0, original_cols = 0;
  int32_t reduced_rows = 0, reduced_cols = 0;
  offset_t reduced_nnz = 0;
  int32_t iterations = 0;
  bool stopped_at_iteration_limit = false;
  bool has_change = false, has_infeasible = false, has_unbounded = false;
  double elapsed_seconds = 0.0, obj_constant_delta = 0.0;
  Record record;
  WorkingLp reduced;          // device arrays (owned iff owns_reduced)
  bool owns_reduced = false;
  std::vector<std::string> trace;
};

void run_presolve(const gpp_lp& input, const gpp_params& p, PresolveOutput& out);

// postsolve_gpu (cpp/src/presolve/gpu_postsolve.cu:535-670): device arrays
// x_org (n0), y_org (m0), z_org (n0) receive the original-space solution.
void run_postsolve(const PresolveOutput& out, const double* x_red, const double* y_red, const double* z_red,
                   const gpp_lp* original, double* x_org, double* y_org, double* z_org);

}  // namespace gpp
