// Diagnostic export of the recovery record (GPU-Preprocessor's
// cpp/include/gpu_preprocessor/presolve/device_recovery.hpp:84,
// export_recovery_record), over gpp_export_maps / gpp_tape_sizes /
// gpp_export_tape.  Postsolve never needs it.
#pragma once

#include <cstdint>
#include <vector>

#include "gpu_preprocessor/detail/status.hpp"
#include "gpu_preprocessor/presolve/presolve_structs.hpp"

namespace gpu_preprocessor::presolve {

// Fills the record's host views: kept row / column maps, fixed values and the
// chronological tape (records in the order they were written).
inline void export_recovery_record(PresolveRecordGpu& record) {
  using gpu_preprocessor::detail::throw_on_status;
  const gpp_summary* s = &record.handle;
  record.row_red2org.assign(static_cast<std::size_t>(record.m1), 0);
  record.col_red2org.assign(static_cast<std::size_t>(record.n1), 0);
  throw_on_status(gpp_export_maps(s, record.row_red2org.data(), record.col_red2org.data()),
                  "export_recovery_record maps");
  std::int64_t records = 0, indices = 0, values = 0, fixed = 0;
  throw_on_status(gpp_tape_sizes(s, &records, &indices, &values, &fixed), "export_recovery_record sizes");
  std::vector<std::int64_t> is(static_cast<std::size_t>(records) + 1), vs(static_cast<std::size_t>(records) + 1);
  PostsolveTape& t = record.tape;
  t.types.assign(static_cast<std::size_t>(records), 0);
  t.indices.assign(static_cast<std::size_t>(indices), 0);
  t.vals.assign(static_cast<std::size_t>(values), 0.0);
  record.fixed_idx.assign(static_cast<std::size_t>(fixed), 0);
  record.fixed_val.assign(static_cast<std::size_t>(fixed), 0.0);
  throw_on_status(gpp_export_tape(s, t.types.data(), is.data(), vs.data(), t.indices.data(), t.vals.data(),
                                  record.fixed_idx.data(), record.fixed_val.data()),
                  "export_recovery_record tape");
  t.index_starts.resize(is.size());
  t.value_starts.resize(vs.size());
  for (std::size_t k = 0; k < is.size(); ++k) {
    t.index_starts[k] = checked_nnz_offset(is[k]);
    t.value_starts[k] = checked_nnz_offset(vs[k]);
  }
}

}  // namespace gpu_preprocessor::presolve
