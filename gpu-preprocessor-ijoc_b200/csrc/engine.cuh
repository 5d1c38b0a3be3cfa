// Internal engine types: device CSR, working LP, deferred plan, live
// statistics, recovery record.  All device data is owned through DBuf or
// explicit ownership flags; everything runs on ctx().stream.
#pragma once

#include <memory>
#include <vector>

#include "common.cuh"

namespace gpp {

struct DevCsr {
  int32_t rows = 0, cols = 0;
  offset_t nnz = 0;
  offset_t* ptr = nullptr;
  int32_t* idx = nullptr;
  double* val = nullptr;
};

// Row-length schedule of one CSR matrix: rows with length <= kShortRow are
// handled one per thread by a pass over all rows; the medium (<= kLongRow)
// and long queues list the remaining rows for warp- and block-per-row work.
struct RowSchedule {
  DBuf<int32_t> medium, long_rows, counts;  // counts[0] medium, counts[1] long
  // Stored schedules only: for every tile of kEntryTile stored entries, the
  // rows that hold its first (x) and last (y) entry.
  DBuf<int2> tile_rows;
  int64_t tiles = 0;
  mutable int sorted = -1;  // rows strictly ascending: -1 not yet checked, else 0 / 1
  const offset_t* ptr = nullptr;
  int32_t rows = -1;
  offset_t nnz = -1;
  uint64_t epoch = 0;
};

// Builds the schedule of `M` by stored length (live_degrees == nullptr) or by
// the given per-row live degree.
void build_schedule(RowSchedule& s, const DevCsr& M, const int32_t* live_degrees, cudaStream_t st);
// Cached stored-length schedule (A and AT slots), invalidated per materialisation.
const RowSchedule& stored_schedule(const DevCsr& M);
void invalidate_schedules();
// Drops any cached schedule of the matrix whose row pointers are `ptr` (called
// when that matrix is freed, since its memory can come back for another).
void forget_schedule(const offset_t* ptr);

struct PostsolveSegment {
  DBuf<int32_t> types;
  DBuf<int64_t> is, vs;   // record offsets into idx / val (count+1 each)
  DBuf<int32_t> idx;
  DBuf<double> val;
  int64_t count = 0, n_idx = 0, n_val = 0;
};

struct FixedSegment {
  DBuf<int32_t> idx;
  DBuf<double> val;
  int64_t count = 0;
};

// Primal recovery of one absolute-value reformulation (reference
// PiecewiseLinearReformulationAbsoluteValuePrimalRecoveryStep,
// presolve_structs.hpp:207-236), on the device.  Column ids are the working
// model's until captured into the record, original ids after.  Restored in
// this order: splits (t, e) <- (t + e, (t - e) / rho); outer pairs
// free <- bound; linked slacks slack <- factor * t; max slacks
// slack <- max(l_slack, max_k factor_k * t_k) per group.
struct AbsValueRecovery {
  int32_t pattern = 0;   // gpp_absolute_value_pattern
  DBuf<int32_t> split_t, split_e;
  DBuf<double> split_rho;
  DBuf<int32_t> pair_bound, pair_free;
  DBuf<int32_t> link_slack, link_t;
  DBuf<double> link_factor;
  DBuf<int32_t> max_slack, max_start, max_t;   // groups; groups + 1; entries
  DBuf<double> max_factor;
  int32_t splits = 0, pairs = 0, links = 0, max_groups = 0, max_entries = 0;
};

// Primal recovery of one variable-pair reformulation (reference
// PiecewiseLinearReformulationVariablePairRecoveryStep, presolve_structs.hpp:243-250):
// x[plus_k] = plus_shift_k + x[root_plus_k], x[minus_k] = minus_shift_k +
// x[root_minus_k], every root value read before any member is written.
struct VarPairRecovery {
  DBuf<int32_t> plus, minus, root_plus, root_minus;
  DBuf<double> plus_shift, minus_shift;
  int32_t count = 0;
};

// Where a primal recovery sits in the tape (reference PrimalRecoveryCheckpoint,
// presolve_structs.hpp:256-266): records at or after `tape_position` are
// replayed (primal pass) before it is applied.
struct RecoveryCheckpoint {
  int32_t kind = 0;        // 0 absolute value, 1 variable pair
  int32_t payload = 0;     // index into Record::absval / Record::varpair
  int64_t tape_position = 0;
};

struct Record {
  int32_t m0 = 0, n0 = 0;
  DBuf<int32_t> rows, cols;   // current index -> original index
  int32_t m = 0, n = 0;
  std::vector<PostsolveSegment> segments;
  std::vector<FixedSegment> fixed;
  std::vector<AbsValueRecovery> absval;
  std::vector<VarPairRecovery> varpair;
  std::vector<RecoveryCheckpoint> timeline;
  int64_t records = 0, indices = 0, values = 0;
};

struct Plan {
  DBuf<uint8_t> keep_row, keep_col;
  DBuf<double> c, l, u, AL, AU;
  double obj_delta = 0.0;
  bool has_change = false, has_row_action = false, has_col_action = false;
  bool has_redundant_row_deletion = false, has_row_deletion = false;
  bool has_infeasible = false, has_unbounded = false;
  // True from a fresh plan (both masks all ones) until the first rule runs
  // on it: a full recount of the live statistics then needs no mask reads.
  bool all_kept = false;
  // When set (scheduled and traced runs), bound strengthening bins the live
  // rows of its activity summary by infinite-term count here: words 0-3 the
  // rows with 0, 1, 2, >= 3 in the minimum activity, 4-7 the maximum.
  uint32_t* inf_hist = nullptr;
  const uint8_t* rule_entry_keep_col = nullptr;
  const double* ref_l = nullptr;
  const double* ref_u = nullptr;
  bool has_new_A = false;
  DevCsr new_A;                  // owned when has_new_A
  std::vector<PostsolveSegment> tape;   // local indices until captured
  std::unique_ptr<AbsValueRecovery> absval;   // set by the absolute-value reformulation
  std::unique_ptr<VarPairRecovery> varpair;   // set by the variable-pair reformulation
};

struct Stats {
  DBuf<int32_t> row_nnz, col_nnz, srow_col, scol_row;
  DBuf<uint8_t> empty_row, singleton_row, empty_col, singleton_col;
  DBuf<double> srow_val, scol_val;
  DBuf<unsigned long long> live_nnz;
  // Incremental refresh: the masks the statistics describe, the rows and
  // columns deleted since, and which of them need their flags recomputed.
  bool valid = false;
  DBuf<uint8_t> seen_row, seen_col, dirty_row, dirty_col;
  DBuf<int32_t> deleted, counters;
};

bool rows_strictly_sorted(const DevCsr& M, cudaStream_t s);

struct WorkingLp {
  DevCsr A, AT;
  double *c = nullptr, *AL = nullptr, *AU = nullptr, *l = nullptr, *u = nullptr;
  double obj = 0.0;
  bool owns = false;
  // Rows of A / AT strictly ascending: 1 yes, 0 no, -1 not checked yet.
  // Compaction keeps a subsequence of every row, so it keeps the property;
  // the transpose builds AT row-sorted.  Checked at most once per matrix.
  mutable int a_sorted = -1, at_sorted = -1;
  bool A_sorted() const {
    if (a_sorted < 0) a_sorted = rows_strictly_sorted(A, ctx().stream) ? 1 : 0;
    return a_sorted != 0;
  }
  bool AT_sorted() const {
    if (at_sorted < 0) at_sorted = rows_strictly_sorted(AT, ctx().stream) ? 1 : 0;
    return at_sorted != 0;
  }
  int32_t m() const { return A.rows; }
  int32_t n() const { return A.cols; }
  void free_owned();
};

// ---- kernel families (host wrappers) ---------------------------------------
// live.cu
void live_stats_side(const DevCsr& M, const uint8_t* keep_outer, const uint8_t* keep_inner,
                     int32_t* degree, uint8_t* empty, uint8_t* singleton, int32_t* support,
                     double* coefficient, unsigned long long* total, cudaStream_t s);
void refresh_stats(Stats& st, const WorkingLp& lp, const Plan& plan);
void allocate_stats(Stats& st, int32_t m, int32_t n);
// Packs {l_j, u_j} of every column (a removed one as the reserved NaN pair).
void pack_bounds(const double* l, const double* u, const uint8_t* keep_col, int32_t n, double2* lu,
                 cudaStream_t s);
void row_activity_summary_packed(const DevCsr& A, const double2* lu, double zero_tol, const uint8_t* keep_row,
                                 const int32_t* live_deg, double* min_fin, double* max_fin, int32_t* min_inf,
                                 int32_t* max_inf, cudaStream_t s);
void row_activity_summary(const DevCsr& A, const double* l, const double* u, double zero_tol,
                          const uint8_t* keep_row, const uint8_t* keep_col, const int32_t* live_deg,
                          double* min_fin, double* max_fin, int32_t* min_inf, int32_t* max_inf,
                          cudaStream_t s);
void row_plain_minmax(const DevCsr& A, const double* l, const double* u, const uint8_t* keep_row,
                      const uint8_t* keep_col, const int32_t* live_deg, double* row_min, double* row_max,
                      cudaStream_t s);
void col_max_abs(const DevCsr& AT, const uint8_t* keep_row, double* out, cudaStream_t s);

// compact.cu
int32_t build_old_to_new(const uint8_t* keep, int32_t n, int32_t* old_to_new, cudaStream_t s);
// Both maps of a materialisation at once (two launches, one readback); returns
// the kept row and column counts.
std::pair<int32_t, int32_t> build_old_to_new_pair(const uint8_t* keep_row, int32_t m, int32_t* row_map,
                                                  const uint8_t* keep_col, int32_t n, int32_t* col_map,
                                                  cudaStream_t s);
// Stable compaction of M's kept rows (outer map) and kept entries (inner map),
// in one pass.  The queued form only launches it: the result's nnz is -1 and
// its index/value arrays hold M.nnz entries until compact_csr_finish applies
// the two result words (kept total, look-back error) read back from
// `result`; so several compactions can share one readback.
DevCsr compact_csr_queued(const DevCsr& M, const int32_t* outer_map, int32_t outer_new, const int32_t* inner_map,
                          int32_t inner_new, cudaStream_t s, int32_t* result, int64_t* profile_record);
void compact_csr_finish(DevCsr& out, const int32_t* result_host, int64_t profile_record);
// Queued and finished at once (one readback).
DevCsr compact_csr(const DevCsr& M, const int32_t* outer_map, int32_t outer_new,
                   const int32_t* inner_map, int32_t inner_new, cudaStream_t s);
// General transpose (histogram, scan, scatter, per-row sort): rows of the
// result list source rows in ascending order.
DevCsr transpose_csr(const DevCsr& M, cudaStream_t s);
// The same transpose into preallocated arrays (t.ptr: M.cols + 1 offsets,
// t.idx / t.val: M.nnz entries).
void transpose_csr_into(const DevCsr& M, const DevCsr& t, cudaStream_t s);
// Checks a CSR's structure on the device: ptr[0] = 0, ptr[rows] = nnz,
// non-decreasing pointers and inner indices in [0, cols).  One readback.
bool csr_structure_valid(const DevCsr& M, cudaStream_t s);
bool rows_strictly_sorted(const DevCsr& M, cudaStream_t s);
void gather_by_map(double* dst, const double* src, const int32_t* old_to_new, int32_t n_old,
                   cudaStream_t s);
void compose_map(int32_t* next, const int32_t* prev, const int32_t* old_to_new, int32_t n_old,
                 cudaStream_t s);
void free_csr(DevCsr& M);

// recovery.cu
void init_record(Record& r, int32_t m, int32_t n);
void globalize_segment(PostsolveSegment& s, const Record& r, cudaStream_t st);
void capture_tape(Record& r, std::vector<PostsolveSegment>& tape);
void append_fixed(Record& r, const uint8_t* keep_col, const uint8_t* prior, const double* l,
                  const double* u, int32_t n);
// Builds a device segment from host-side packed arrays (records laid out
// contiguously); used by rules that pack on the device and know the counts.
PostsolveSegment make_segment(int64_t count, int64_t n_idx, int64_t n_val);
// Moves an absolute-value recovery into the record (column ids made
// original through r.cols) with a checkpoint at the current tape length.
void capture_absolute_value(Record& r, AbsValueRecovery&& step);
void capture_variable_pair(Record& r, VarPairRecovery&& step);

// rules_*.cu
// The first-stage detections of the first four Cleanup rules at once, with
// one readback: returns the kProbe* bits of `rules` whose rule may change the
// plan.  A rule whose bit comes back clear would return at its first check
// without changing anything, as long as the plan is the probed one.
constexpr uint32_t kProbeFixed = 1, kProbeEmptyColumns = 2, kProbeEmptyRows = 4, kProbeSingletonRows = 8;
uint32_t cleanup_probe(const Plan& plan, const WorkingLp& lp, const Stats& stats, const gpp_params& p, uint32_t rules);
void rule_fixed_variables(Plan& plan, const WorkingLp& lp, const gpp_params& p);
void rule_empty_columns(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
void rule_empty_rows(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
void rule_singleton_rows(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
void rule_singleton_columns(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
void rule_bound_strengthening(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
void rule_redundant_rows(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
void rule_dual_fix(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
// rules_startup.cu: structure-specific Startup rules.
void rule_column_domination(Plan& plan, const WorkingLp& lp, const gpp_params& p);
void rule_two_row_variable_elimination(Plan& plan, const WorkingLp& lp, const gpp_params& p);
void rule_zero_cost_product_variables(Plan& plan, const WorkingLp& lp, const gpp_params& p);
void rule_parallel_rows(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
void rule_parallel_columns(Plan& plan, const WorkingLp& lp, const Stats& s, const gpp_params& p);
void rule_doubleton_equations(Plan& plan, const WorkingLp& lp, const gpp_params& p);
// rules_pwl_abs.cu: piecewise-linear reformulation of absolute values.
// The prefix screen (rows 0-3 look like one of the three layouts) gates the
// rule as the reference's does.
bool absolute_value_prefix_screen(const WorkingLp& lp);
void rule_absolute_value(Plan& plan, const WorkingLp& lp, const gpp_params& p);
// rules_pwl_pair.cu: piecewise-linear reformulation of variable pairs
// (epigraph, else shifted antipodal).
void rule_variable_pair(Plan& plan, const WorkingLp& lp, const gpp_params& p);

// Row-wise shift sum_j a_ij * v_j over kept rows and selected columns, in
// ascending column order (deterministic replacement of atomicAdd shifts).
// With `radius`, sums |a_ij| * radius_j over selected columns with radius > 0.
void row_gather_shift(const DevCsr& A, const DevCsr& AT, const uint8_t* keep_row, const uint8_t* selected,
                      const double* value, const double* radius, double* out, cudaStream_t s);
// Canonical objective sum of contrib over the rule-entry domain.
double domain_objective(const double* contrib, const uint8_t* entry_keep, int32_t n, cudaStream_t s);

}  // namespace gpp
