// Device postsolve of the C++ layer (GPU-Preprocessor's
// cpp/include/gpu_preprocessor/presolve/gpu_postsolve.hpp:20-31 and
// cpp/src/presolve/gpu_postsolve.cu:527-560), over gpp_postsolve_device.
#pragma once

#include <stdexcept>
#include <vector>

#include "gpu_preprocessor/detail/status.hpp"
#include "gpu_preprocessor/presolve/presolve_structs.hpp"

namespace gpu_preprocessor::presolve {

// Maps a reduced solution (device arrays of reduced_cols / reduced_rows /
// reduced_cols entries; any may be nullptr) back to the presolve input.  The
// result's x_org / y_org / z_org are device arrays of n0 / m0 / n0 entries
// allocated here; the caller releases them with cudaFree.  With
// original_model, row duals are completed by the dual projection the record
// asks for; without it only the primal side is recovered exactly.
// original_l (device, n0 entries) bounds the absolute-value reformulation's
// max slacks below; when it is null the original model's l is used.
inline GpuPostsolveResult postsolve_gpu(double* x_red, double* y_red, double* z_red, const PresolveRecordGpu& record,
                                        const LPInfoGpu* original_model, const double* original_l = nullptr) {
  using gpu_preprocessor::detail::throw_on_status;
  GpuPostsolveResult r;
  r.n0 = record.n0;
  r.m0 = record.m0;
  auto alloc = [](double** p, std::int32_t n, const char* what) {
    if (n > 0) throw_on_status(gpp_device_alloc(reinterpret_cast<void**>(p), sizeof(double) * std::size_t(n)), what);
  };
  try {
    alloc(&r.x_org, r.n0, "postsolve_gpu x_org");
    alloc(&r.z_org, r.n0, "postsolve_gpu z_org");
    alloc(&r.y_org, r.m0, "postsolve_gpu y_org");
    throw_on_status(gpp_postsolve_device_lower(x_red, y_red, z_red, &record.handle, detail::as_c(original_model),
                                               original_l, r.x_org, r.y_org, r.z_org),
                    "postsolve_gpu");
  } catch (...) {
    gpp_device_free(r.x_org);
    gpp_device_free(r.y_org);
    gpp_device_free(r.z_org);
    throw;
  }
  return r;
}

inline GpuPostsolveResult postsolve_gpu(double* x_red, double* y_red, double* z_red, const PresolveRecordGpu& record,
                                        const double* original_l = nullptr) {
  return postsolve_gpu(x_red, y_red, z_red, record, nullptr, original_l);
}

// The absolute-value recovery steps alone, applied last to first to the
// device vector x_org (gpu_postsolve.hpp:12-18 of the reference).
inline void postsolve_restore_piecewise_linear_reformulation_absolute_value_gpu(
    double* x_org, const std::vector<PiecewiseLinearReformulationAbsoluteValuePrimalRecoveryStep>& recoveries,
    const double* original_l = nullptr) {
  using gpu_preprocessor::detail::throw_on_status;
  struct Flat {
    std::vector<std::int32_t> st, se, pb, pf, ls, lt, ms, mstart{0}, mt;
    std::vector<double> sr, lf, mf;
  };
  std::vector<Flat> flat(recoveries.size());
  std::vector<gpp_absolute_value_recovery> steps(recoveries.size());
  for (std::size_t k = 0; k < recoveries.size(); ++k) {
    const auto& r = recoveries[k];
    Flat& f = flat[k];
    for (const auto& x : r.splits) { f.st.push_back(x.t_col); f.se.push_back(x.e_col); f.sr.push_back(x.rho); }
    for (const auto& x : r.outer_pairs) { f.pb.push_back(x.bound_col); f.pf.push_back(x.free_col); }
    for (const auto& x : r.linked_slacks) {
      f.ls.push_back(x.slack_col);
      f.lt.push_back(x.t_col);
      f.lf.push_back(x.factor);
    }
    for (const auto& g : r.max_slacks) {
      if (g.t_cols.size() != g.factors.size())
        throw std::runtime_error("piecewise_linear_reformulation_absolute_value max-slack recovery has mismatched payloads");
      f.ms.push_back(g.slack_col);
      f.mt.insert(f.mt.end(), g.t_cols.begin(), g.t_cols.end());
      f.mf.insert(f.mf.end(), g.factors.begin(), g.factors.end());
      f.mstart.push_back(static_cast<std::int32_t>(f.mt.size()));
    }
    steps[k] = gpp_absolute_value_recovery{
        r.pattern == "l1_split_3row" ? GPP_ABS_L1_SPLIT : r.pattern == "graph_l1_substitution" ? GPP_ABS_GRAPH_L1
                                                                                             : GPP_ABS_OUTER_PAIR,
        static_cast<std::int32_t>(f.st.size()), f.st.data(), f.se.data(), f.sr.data(),
        static_cast<std::int32_t>(f.pb.size()), f.pb.data(), f.pf.data(),
        static_cast<std::int32_t>(f.ls.size()), f.ls.data(), f.lt.data(), f.lf.data(),
        static_cast<std::int32_t>(f.ms.size()), f.ms.data(), f.mstart.data(), f.mt.data(), f.mf.data()};
  }
  throw_on_status(gpp_restore_absolute_value(x_org, steps.data(), static_cast<std::int32_t>(steps.size()), original_l),
                  "postsolve_restore_piecewise_linear_reformulation_absolute_value_gpu");
}

}  // namespace gpu_preprocessor::presolve
