// Device postsolve of the C++ layer (GPU-Preprocessor's
// cpp/include/gpu_preprocessor/presolve/gpu_postsolve.hpp:20-31 and
// cpp/src/presolve/gpu_postsolve.cu:527-560), over gpp_postsolve_device.
#pragma once

#include "gpu_preprocessor/detail/status.hpp"
#include "gpu_preprocessor/presolve/presolve_structs.hpp"

namespace gpu_preprocessor::presolve {

// Maps a reduced solution (device arrays of reduced_cols / reduced_rows /
// reduced_cols entries; any may be nullptr) back to the presolve input.  The
// result's x_org / y_org / z_org are device arrays of n0 / m0 / n0 entries
// allocated here; the caller releases them with cudaFree.  With
// original_model, row duals are completed by the dual projection the record
// asks for; without it only the primal side is recovered exactly.
// original_l is consulted by the reference only for the recoveries of the
// structure-specific reformulations, which this engine never records.
inline GpuPostsolveResult postsolve_gpu(double* x_red, double* y_red, double* z_red, const PresolveRecordGpu& record,
                                        const LPInfoGpu* original_model, const double* original_l = nullptr) {
  using gpu_preprocessor::detail::throw_on_status;
  (void)original_l;
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
    throw_on_status(gpp_postsolve_device(x_red, y_red, z_red, &record.handle, detail::as_c(original_model), r.x_org,
                                         r.y_org, r.z_org),
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

}  // namespace gpu_preprocessor::presolve
