// Public structs of the presolve layer, over gpp.h.
//
// Names, field order and defaults follow GPU-Preprocessor's
// cpp/include/gpu_preprocessor/presolve/presolve_structs.hpp (PresolveParams
// :28-158, DeviceCsrMatrix :160-167, LPInfoGpu :169-180, PostsolveReductionType
// :268-282, PostsolveTape :317-331, PresolveRecordGpu :338-368,
// GpuPostsolveResult :370-376), so code written against the reference compiles
// unchanged.  DeviceCsrMatrix and LPInfoGpu are layout-identical to gpp_csr and
// gpp_lp (checked below), so they cross the C ABI without copies.
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include "gpp.h"
#include "gpu_preprocessor/offset.hpp"

namespace gpu_preprocessor::presolve {

enum class PiecewiseLinearReformulationAbsoluteValueResidualBoundMode : std::uint8_t {
  PreserveFinite = 0,
  StrictFreeOnly = 1,
  LegacyWideAsFree = 2,
};

// One line per PresolveParams field: type, name, default.  The struct below
// and the conversion to gpp_params are both generated from this list, so the
// two cannot drift apart.
#define GPP_PRESOLVE_PARAM_FIELDS(X)                                                                       \
  X(int, max_iters, 512)                                                                                   \
  X(double, max_time, std::numeric_limits<double>::infinity())                                            \
  X(bool, verbose, false)                                                                                  \
  X(bool, record_postsolve_tape, true)                                                                     \
  X(bool, record_postsolve_tape_cpu, false)                                                                \
  X(bool, enable_presolve, true)                                                                           \
  X(bool, enable_folding, true)                                                                            \
  X(double, folding_tolerance, 1.0e-8)                                                                     \
  X(double, feasibility_tol, 1.0e-6)                                                                       \
  X(double, bound_tol, 1.0e-6)                                                                             \
  X(double, zero_tol, 1.0e-10)                                                                             \
  X(double, bound_strengthening_upper_relaxation_factor, 1.0)                                              \
  X(int, bound_strengthening_max_rounds, 64)                                                               \
  X(int, bound_strengthening_max_bound_only_rounds, 64)                                                    \
  X(bool, bound_strengthening_preserve_free_zero_cost, true)                                               \
  X(int, doubleton_equations_max_fill_in_proxy, 96)                                                        \
  X(bool, doubleton_equations_scan, true)                                                                  \
  X(int, doubleton_equations_min_selected_per_batch, 256)                                                  \
  X(double, doubleton_equations_min_selected_ratio, 0.005)                                                 \
  X(int, doubleton_equations_max_batch_rounds, 0)                                                          \
  X(double, doubleton_equations_max_time, 0.0)                                                             \
  X(bool, enable_infeasible_and_fixed_variables, true)                                                     \
  X(bool, enable_empty_rows, true)                                                                         \
  X(bool, enable_singleton_rows, true)                                                                     \
  X(bool, enable_infeasible_and_redundant_rows, true)                                                      \
  X(bool, enable_bound_strengthening, true)                                                                \
  X(bool, enable_parallel_rows, true)                                                                      \
  X(bool, enable_empty_columns, true)                                                                      \
  X(bool, enable_singleton_columns, true)                                                                  \
  X(bool, enable_doubleton_equations, true)                                                                \
  X(bool, enable_dual_fix, true)                                                                           \
  X(int, dual_fix_max_nonzero_cost_col_degree, 128)                                                        \
  X(bool, enable_parallel_columns, true)                                                                   \
  X(double, parallel_columns_max_abs_ratio, 2.0)                                                           \
  X(int, parallel_columns_scale_guard_max_group_size, 4)                                                   \
  X(int, parallel_columns_scale_guard_min_groups, 128)                                                     \
  X(bool, enable_structure_specific_rules, true)                                                           \
  X(bool, enable_two_row_variable_elimination, true)                                                       \
  X(int, two_row_variable_elimination_max_row_nnz, 8)                                                      \
  X(double, two_row_variable_elimination_safety_tol, 1.0e-8)                                               \
  X(int, two_row_variable_elimination_min_candidates, 128)                                                 \
  X(double, two_row_variable_elimination_min_candidate_ratio, 0.01)                                        \
  X(bool, enable_zero_cost_product_variables, true)                                                        \
  X(int, zero_cost_product_variables_min_candidates, 128)                                                  \
  X(double, zero_cost_product_variables_min_candidate_ratio, 0.01)                                         \
  X(bool, enable_piecewise_linear_reformulation_variable_pair, true)                                       \
  X(int, piecewise_linear_reformulation_variable_pair_epigraph_probe_pairs, 256)                           \
  X(int, piecewise_linear_reformulation_variable_pair_epigraph_min_pairs, 4096)                            \
  X(double, piecewise_linear_reformulation_variable_pair_epigraph_min_potential_gain, 0.20)                \
  X(double, piecewise_linear_reformulation_variable_pair_epigraph_min_actual_gain, 0.20)                   \
  X(int, piecewise_linear_reformulation_variable_pair_epigraph_max_tail_cols, 8)                           \
  X(int, piecewise_linear_reformulation_variable_pair_epigraph_max_quotient_terms_per_row, 5)              \
  X(int, piecewise_linear_reformulation_variable_pair_shifted_antipodal_probe_pairs, 256)                  \
  X(int, piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs, 4096)                   \
  X(double, piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_potential_gain, 0.20)       \
  X(double, piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_actual_gain, 0.20)          \
  X(int, piecewise_linear_reformulation_variable_pair_shifted_antipodal_max_quotient_terms_per_row, 6)     \
  X(bool, enable_column_domination, true)                                                                  \
  X(int, column_domination_probe_rows, 64)                                                                 \
  X(int, column_domination_probe_cols, 256)                                                                \
  X(int, column_domination_probe_nnz, 256)                                                                 \
  X(int, column_domination_min_fixed_cols, 4096)                                                           \
  X(double, column_domination_min_candidate_ratio, 0.20)                                                   \
  X(bool, enable_piecewise_linear_reformulation_absolute_value, true)                                      \
  X(PiecewiseLinearReformulationAbsoluteValueResidualBoundMode,                                            \
    piecewise_linear_reformulation_absolute_value_residual_bound_mode,                                     \
    PiecewiseLinearReformulationAbsoluteValueResidualBoundMode::PreserveFinite)                            \
  X(double, piecewise_linear_reformulation_absolute_value_residual_bound_as_free_min, 1.0e8)               \
  X(bool, enable_redundant_variable_bounds, false)                                                         \
  X(bool, enable_startup, true)                                                                            \
  X(std::int64_t, bound_strengthening_bound_only_nnz_round_budget, 8000000)

// The structure-specific startup rules (column domination, two-row variable
// elimination, zero-cost product variables, the piecewise-linear
// reformulations, redundant variable bounds) are accepted for source
// compatibility; this engine does not run them.
struct PresolveParams {
#define GPP_DECLARE_FIELD(type, name, value) type name = value;
  GPP_PRESOLVE_PARAM_FIELDS(GPP_DECLARE_FIELD)
#undef GPP_DECLARE_FIELD
};

namespace detail {
inline gpp_params to_c(const PresolveParams& p) {
  gpp_params c;
  gpp_default_params(&c);
#define GPP_COPY_FIELD(type, name, value) c.name = static_cast<decltype(c.name)>(p.name);
  GPP_PRESOLVE_PARAM_FIELDS(GPP_COPY_FIELD)
#undef GPP_COPY_FIELD
  return c;
}
}  // namespace detail

struct DeviceCsrMatrix {
  std::int32_t rows = 0;
  std::int32_t cols = 0;
  NnzOffset nnz = 0;
  NnzOffset* rowPtr = nullptr;
  std::int32_t* colVal = nullptr;
  double* nzVal = nullptr;
};

struct LPInfoGpu {
  DeviceCsrMatrix A;
  DeviceCsrMatrix AT;
  double* c = nullptr;
  double* AL = nullptr;
  double* AU = nullptr;
  double* l = nullptr;
  double* u = nullptr;
  double obj_constant = 0.0;
  NnzOffset AT_leading_slack = 0;
  NnzOffset* AT_slack_after = nullptr;
};

static_assert(sizeof(DeviceCsrMatrix) == sizeof(gpp_csr) &&
                  offsetof(DeviceCsrMatrix, nnz) == offsetof(gpp_csr, nnz) &&
                  offsetof(DeviceCsrMatrix, rowPtr) == offsetof(gpp_csr, rowPtr) &&
                  offsetof(DeviceCsrMatrix, nzVal) == offsetof(gpp_csr, nzVal),
              "DeviceCsrMatrix must match gpp_csr");
static_assert(sizeof(LPInfoGpu) == sizeof(gpp_lp) && offsetof(LPInfoGpu, AT) == offsetof(gpp_lp, AT) &&
                  offsetof(LPInfoGpu, c) == offsetof(gpp_lp, c) && offsetof(LPInfoGpu, u) == offsetof(gpp_lp, u) &&
                  offsetof(LPInfoGpu, obj_constant) == offsetof(gpp_lp, obj_constant) &&
                  offsetof(LPInfoGpu, AT_slack_after) == offsetof(gpp_lp, AT_slack_after),
              "LPInfoGpu must match gpp_lp");

namespace detail {
inline const gpp_lp* as_c(const LPInfoGpu* lp) { return reinterpret_cast<const gpp_lp*>(lp); }
inline DeviceCsrMatrix from_c(const gpp_csr& m) { return {m.rows, m.cols, m.nnz, m.rowPtr, m.colVal, m.nzVal}; }
inline LPInfoGpu from_c(const gpp_lp& lp) {
  LPInfoGpu out;
  out.A = from_c(lp.A);
  out.AT = from_c(lp.AT);
  out.c = lp.c;
  out.AL = lp.AL;
  out.AU = lp.AU;
  out.l = lp.l;
  out.u = lp.u;
  out.obj_constant = lp.obj_constant;
  out.AT_leading_slack = lp.AT_leading_slack;
  out.AT_slack_after = lp.AT_slack_after;
  return out;
}
}  // namespace detail

enum class PostsolveReductionType : std::int32_t {
  FixedVariable = 0,
  InfiniteBoundDualFix = 1,
  SingletonColumnSubstitution = 2,
  ParallelColumn = 3,
  ParallelRow = 4,
  DeletedRow = 5,
  RowLowerBoundChange = 8,
  RowUpperBoundChange = 9,
  RowDualShift = 10,
  VariableBoundChange = 11,
  RowImpliedBoundChange = 12,
  DoubletonEquation = 13,
  FmeCol = 14,
};

// Primal recovery of the absolute-value reformulation (the reference's
// presolve_structs.hpp:207-236): host views filled by export_recovery_record
// and the input of postsolve_restore_piecewise_linear_reformulation_absolute_value_gpu.
struct PiecewiseLinearReformulationAbsoluteValueSplitRecovery {
  std::int32_t t_col = -1;
  std::int32_t e_col = -1;
  double rho = 1.0;
};

struct AbsoluteValueOuterPairRecovery {
  std::int32_t bound_col = -1;
  std::int32_t free_col = -1;
};

struct AbsoluteValueLinkedSlackRecovery {
  std::int32_t slack_col = -1;
  std::int32_t t_col = -1;
  double factor = 0.0;
};

struct AbsoluteValueMaxSlackRecovery {
  std::int32_t slack_col = -1;
  std::vector<std::int32_t> t_cols;
  std::vector<double> factors;
};

struct PiecewiseLinearReformulationAbsoluteValuePrimalRecoveryStep {
  std::string pattern;
  std::vector<PiecewiseLinearReformulationAbsoluteValueSplitRecovery> splits;
  std::vector<AbsoluteValueOuterPairRecovery> outer_pairs;
  std::vector<AbsoluteValueLinkedSlackRecovery> linked_slacks;
  std::vector<AbsoluteValueMaxSlackRecovery> max_slacks;
};

// Primal recovery of the variable-pair reformulation (presolve_structs.hpp:243-250).
struct PiecewiseLinearReformulationVariablePairRecoveryStep {
  std::vector<std::int32_t> plus_cols;
  std::vector<std::int32_t> minus_cols;
  std::vector<std::int32_t> root_plus_cols;
  std::vector<std::int32_t> root_minus_cols;
  std::vector<double> plus_shift;
  std::vector<double> minus_shift;
};

// Where a primal recovery sits among the tape records (presolve_structs.hpp:252-266).
enum class PrimalRecoveryKind : std::uint8_t {
  PiecewiseLinearReformulationAbsoluteValue = 0,
  PiecewiseLinearReformulationVariablePair = 1,
};

struct PrimalRecoveryCheckpoint {
  PrimalRecoveryKind kind = PrimalRecoveryKind::PiecewiseLinearReformulationAbsoluteValue;
  NnzOffset payload_index = -1;
  NnzOffset tape_position = 0;
};

// Host view of the recovery tape, filled only by export_recovery_record.
// Postsolve never needs it: the tape stays on the device.
struct PostsolveTape {
  std::vector<std::int32_t> types;
  std::vector<NnzOffset> index_starts{0};
  std::vector<NnzOffset> value_starts{0};
  std::vector<std::int32_t> indices;
  std::vector<double> vals;
};

// The GPU-resident postsolve record.  Its device state is released by
// free_summary / free_gpu_presolve_reduced_lp, never by a destructor.  Like
// the reference's record it can be moved but not copied, so exactly one
// summary holds the handle; a moved-from record holds none and freeing it is
// a no-op.  The host vectors are empty until export_recovery_record fills them.
struct PresolveRecordGpu {
  PresolveRecordGpu() = default;
  PresolveRecordGpu(const PresolveRecordGpu&) = delete;
  PresolveRecordGpu& operator=(const PresolveRecordGpu&) = delete;
  PresolveRecordGpu(PresolveRecordGpu&& o) noexcept { *this = static_cast<PresolveRecordGpu&&>(o); }
  PresolveRecordGpu& operator=(PresolveRecordGpu&& o) noexcept {
    if (this != &o) {
      m0 = o.m0; n0 = o.n0; m1 = o.m1; n1 = o.n1;
      row_red2org.swap(o.row_red2org); col_red2org.swap(o.col_red2org);
      fixed_idx.swap(o.fixed_idx); fixed_val.swap(o.fixed_val);
      obj_constant_old = o.obj_constant_old; obj_constant_new = o.obj_constant_new;
      tape.types.swap(o.tape.types); tape.index_starts.swap(o.tape.index_starts);
      tape.value_starts.swap(o.tape.value_starts); tape.indices.swap(o.tape.indices);
      tape.vals.swap(o.tape.vals);
      piecewise_linear_reformulation_absolute_value_recoveries.swap(
          o.piecewise_linear_reformulation_absolute_value_recoveries);
      piecewise_linear_reformulation_variable_pair_recoveries.swap(
          o.piecewise_linear_reformulation_variable_pair_recoveries);
      primal_recovery_timeline.swap(o.primal_recovery_timeline);
      handle = o.handle;
      o.handle = gpp_summary{};
    }
    return *this;
  }

  std::int32_t m0 = 0;
  std::int32_t n0 = 0;
  std::int32_t m1 = 0;
  std::int32_t n1 = 0;
  std::vector<std::int32_t> row_red2org;
  std::vector<std::int32_t> col_red2org;
  std::vector<std::int32_t> fixed_idx;
  std::vector<double> fixed_val;
  double obj_constant_old = 0.0;
  double obj_constant_new = 0.0;
  PostsolveTape tape;
  std::vector<PiecewiseLinearReformulationAbsoluteValuePrimalRecoveryStep>
      piecewise_linear_reformulation_absolute_value_recoveries;
  std::vector<PiecewiseLinearReformulationVariablePairRecoveryStep>
      piecewise_linear_reformulation_variable_pair_recoveries;
  std::vector<PrimalRecoveryCheckpoint> primal_recovery_timeline;
  gpp_summary handle{};  // the C-ABI summary whose record this is
};

// Device vectors in original order, allocated by postsolve_gpu; the caller
// releases them with cudaFree.
struct GpuPostsolveResult {
  double* x_org = nullptr;
  double* y_org = nullptr;
  double* z_org = nullptr;
  std::int32_t n0 = 0;
  std::int32_t m0 = 0;
};

}  // namespace gpu_preprocessor::presolve
