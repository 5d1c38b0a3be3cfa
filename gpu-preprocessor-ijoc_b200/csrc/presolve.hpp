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

// ---- round schedule ---------------------------------------------------------
// One round is one step of the phase machine (Cleanup, Propagation,
// Aggregation or Parallel).  Six rules can be gated per round.
enum GatedRule : int {
  kGateSingletonColumns = 0,
  kGateBoundStrengthening = 1,
  kGateRedundantRowsDualFix = 2,
  kGateDoubleton = 3,
  kGateParallelRows = 4,
  kGateParallelColumns = 5,
  kGatedRules = 6
};
constexpr int kScheduleFeatures = 32;

// What the host knows at the start of a round, normalised to about [0, 1]:
//  0-3   phase one-hot (Cleanup, Propagation, Aggregation, Parallel)
//  4     round index / 32
//  5     live nnz / initial nnz
//  6, 7  nnz removed by the previous round and the one before, / initial nnz
//  8-13  per gated rule: 1 if it changed the model the last time it ran
//  14-19 per gated rule: rounds since it last ran / 16 (1 if never)
//  20    consecutive bound-only propagation rounds / 8
//  21    log10(initial nnz) / 8
//  22    share of the initial nnz removed so far
//  23    kept rows / initial rows (as of the last materialisation)
//  24-27 share of the live rows whose latest activity summary (the last
//        bound-strengthening sweep) counts 0, 1, 2 or >= 3 infinite terms
//        in the minimum activity; all zero before the first sweep
//  28-31 the same for the maximum activity
struct RoundRecord {
  int32_t phase = 0;          // 0 Cleanup, 1 Propagation, 2 Aggregation, 3 Parallel
  int32_t iteration = 0;
  uint32_t ran = 0;           // bit per gated rule that ran this round
  uint32_t changed = 0;       // bit per gated rule that changed the model
  int64_t nnz_before = 0, nnz_after = 0;
  float features[kScheduleFeatures] = {};
};

// Decides, per round, which gated rules to skip and whether to stop; the plain
// phase machine is what runs when no policy is given.
struct SchedulePolicy {
  virtual ~SchedulePolicy() = default;
  // Returns the skip mask (bit per gated rule); sets *stop to end presolve.
  virtual uint32_t decide(const float* features, bool* stop) = 0;
};

void run_presolve(const gpp_lp& input, const gpp_params& p, PresolveOutput& out,
                  SchedulePolicy* policy = nullptr, std::vector<RoundRecord>* trace = nullptr);

// postsolve_gpu (cpp/src/presolve/gpu_postsolve.cu:535-670): device arrays
// x_org (n0), y_org (m0), z_org (n0) receive the original-space solution.
// Applies one absolute-value primal recovery to the device vector x
// (original order); `lower` (device, may be null) bounds the max slacks.
void restore_absolute_value(double* x, const AbsValueRecovery& r, const double* lower, cudaStream_t st);
// Applies one variable-pair primal recovery to x.
void restore_variable_pair(double* x, const VarPairRecovery& r, cudaStream_t st);
// `lower` bounds the absolute-value max slacks (original->l when null).
void run_postsolve(const PresolveOutput& out, const double* x_red, const double* y_red, const double* z_red,
                   const gpp_lp* original, double* x_org, double* y_org, double* z_org,
                   const double* lower = nullptr);

}  // namespace gpp
