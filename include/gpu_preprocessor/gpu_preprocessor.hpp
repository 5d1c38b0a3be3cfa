// The plain pipeline of the C++ layer: preprocess / postprocess /
// free_summary, with the type aliases of GPU-Preprocessor's
// cpp/include/gpu_preprocessor/gpu_preprocessor.hpp:8-41.  Link against
// libgpp_b200.so; every call goes through the C ABI in gpp.h.
#pragma once

#include "gpu_preprocessor/folding/folding.hpp"
#include "gpu_preprocessor/presolve/device_recovery.hpp"
#include "gpu_preprocessor/presolve/gpu_postsolve.hpp"

namespace gpu_preprocessor {

using Parameters = presolve::PresolveParams;
using DeviceLp = presolve::LPInfoGpu;
using Summary = folding::FoldingPipelineSummary;
using Solution = folding::UnfoldedSolutionHost;

// Folding, then presolve.  The input stays caller-owned and unchanged; keep it
// and the summary alive until postprocess.  The reduced model may borrow the
// input's arrays.
inline Summary preprocess(const DeviceLp& input, const Parameters& params = {}) {
  return folding::run_gpu_presolve_with_folding(input, params, true, true);
}

// x, y, z: device arrays in reduced order (reduced_cols, reduced_rows,
// reduced_cols entries).  Returns host vectors in original order; dual
// convention c - A^T y - z = 0.
inline Solution postprocess(double* x, double* y, double* z, const Summary& summary, const DeviceLp& original) {
  return folding::postsolve_and_unfold_to_host(x, y, z, summary, &original);
}

// Releases everything the summary holds; a second call is a no-op.
inline void free_summary(Summary& summary) {
  gpp_free_summary(&summary.presolve.record.handle);
  summary = Summary{};
}

}  // namespace gpu_preprocessor
