// Diagnostic export of the recovery record (GPU-Preprocessor's
// cpp/include/gpu_preprocessor/presolve/device_recovery.hpp:84,
// export_recovery_record), over gpp_export_maps / gpp_tape_sizes /
// gpp_export_tape / gpp_recovery_checkpoints / gpp_export_absolute_value.
// Postsolve never needs it.
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
  // Primal-recovery checkpoints and the absolute-value payloads.
  std::int32_t count = 0;
  throw_on_status(gpp_recovery_checkpoints(s, &count, nullptr, nullptr, nullptr), "export_recovery_record checkpoints");
  std::vector<std::int32_t> kinds(static_cast<std::size_t>(count)), payloads(static_cast<std::size_t>(count));
  std::vector<std::int64_t> positions(static_cast<std::size_t>(count));
  throw_on_status(gpp_recovery_checkpoints(s, &count, kinds.data(), payloads.data(), positions.data()),
                  "export_recovery_record checkpoints");
  record.primal_recovery_timeline.clear();
  record.piecewise_linear_reformulation_absolute_value_recoveries.clear();
  record.piecewise_linear_reformulation_variable_pair_recoveries.clear();
  for (std::int32_t k = 0; k < count; ++k) {
    record.primal_recovery_timeline.push_back({static_cast<PrimalRecoveryKind>(kinds[std::size_t(k)]),
                                               checked_nnz_offset(payloads[std::size_t(k)]),
                                               checked_nnz_offset(positions[std::size_t(k)])});
    if (kinds[std::size_t(k)] == 1) {
      std::int32_t n = 0;
      throw_on_status(gpp_variable_pair_size(s, payloads[std::size_t(k)], &n), "export_recovery_record sizes");
      PiecewiseLinearReformulationVariablePairRecoveryStep step;
      step.plus_cols.resize(std::size_t(n));
      step.minus_cols.resize(std::size_t(n));
      step.root_plus_cols.resize(std::size_t(n));
      step.root_minus_cols.resize(std::size_t(n));
      step.plus_shift.resize(std::size_t(n));
      step.minus_shift.resize(std::size_t(n));
      throw_on_status(gpp_export_variable_pair(s, payloads[std::size_t(k)], step.plus_cols.data(),
                                               step.minus_cols.data(), step.root_plus_cols.data(),
                                               step.root_minus_cols.data(), step.plus_shift.data(),
                                               step.minus_shift.data()),
                      "export_recovery_record variable pair");
      record.piecewise_linear_reformulation_variable_pair_recoveries.push_back(std::move(step));
      continue;
    }
    if (kinds[std::size_t(k)] != 0) continue;
    std::int32_t z[6];
    throw_on_status(gpp_absolute_value_sizes(s, payloads[std::size_t(k)], z), "export_recovery_record sizes");
    std::vector<std::int32_t> st(z[1]), se(z[1]), pb(z[2]), pf(z[2]), ls(z[3]), lt(z[3]), ms(z[4]),
        mstart(std::size_t(z[4]) + 1), mt(z[5]);
    std::vector<double> sr(z[1]), lf(z[3]), mf(z[5]);
    throw_on_status(gpp_export_absolute_value(s, payloads[std::size_t(k)], st.data(), se.data(), sr.data(), pb.data(),
                                              pf.data(), ls.data(), lt.data(), lf.data(), ms.data(), mstart.data(),
                                              mt.data(), mf.data()),
                    "export_recovery_record absolute value");
    PiecewiseLinearReformulationAbsoluteValuePrimalRecoveryStep step;
    step.pattern = z[0] == GPP_ABS_L1_SPLIT ? "l1_split_3row"
                   : z[0] == GPP_ABS_GRAPH_L1 ? "graph_l1_substitution"
                                              : "outer_pair_linked_l1";
    for (std::int32_t i = 0; i < z[1]; ++i) step.splits.push_back({st[std::size_t(i)], se[std::size_t(i)], sr[std::size_t(i)]});
    for (std::int32_t i = 0; i < z[2]; ++i) step.outer_pairs.push_back({pb[std::size_t(i)], pf[std::size_t(i)]});
    for (std::int32_t i = 0; i < z[3]; ++i)
      step.linked_slacks.push_back({ls[std::size_t(i)], lt[std::size_t(i)], lf[std::size_t(i)]});
    for (std::int32_t g = 0; g < z[4]; ++g) {
      AbsoluteValueMaxSlackRecovery m;
      m.slack_col = ms[std::size_t(g)];
      m.t_cols.assign(mt.begin() + mstart[std::size_t(g)], mt.begin() + mstart[std::size_t(g) + 1]);
      m.factors.assign(mf.begin() + mstart[std::size_t(g)], mf.begin() + mstart[std::size_t(g) + 1]);
      step.max_slacks.push_back(std::move(m));
    }
    record.piecewise_linear_reformulation_absolute_value_recoveries.push_back(std::move(step));
  }
}

}  // namespace gpu_preprocessor::presolve
