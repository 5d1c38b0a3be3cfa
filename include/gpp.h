/*
 * gpp.h -- C ABI of the B200-native LP presolve / postsolve engine.
 *
 * This is the drop-in boundary for the plain presolve path of GPU-Preprocessor.
 * Every entry point takes plain pointers and sizes (device pointers where the
 * reference takes device pointers), returns an int status (0 = success) and
 * never throws.  The C++ API of the reference (namespaces gpu_preprocessor,
 * gpu_preprocessor::presolve, gpu_preprocessor::folding) is provided as a
 * header-only layer over these functions in include/gpu_preprocessor/.
 *
 * Layouts follow the reference's public structs:
 *   gpp_csr      <-> DeviceCsrMatrix   (cpp/include/gpu_preprocessor/presolve/presolve_structs.hpp:160-167)
 *   gpp_lp       <-> LPInfoGpu         (presolve_structs.hpp:169-180)
 *   gpp_params   <-> PresolveParams    (presolve_structs.hpp:28-158)
 *   gpp_summary  <-> GpuPresolveSummary + FoldingPipelineSummary
 *                                      (presolve/gpu_presolve.hpp:14-30, folding/folding_structs.hpp:94-109)
 * Offsets (NnzOffset) are int32, the reference's default ABI
 * (cpp/include/gpu_preprocessor/offset.hpp:12-19).
 */
#ifndef GPP_H_
#define GPP_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GPP_API __attribute__((visibility("default")))
#else
#define GPP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gpp_offset;

/* Status codes.  Model status (infeasible / unbounded) is reported in the
 * summary, not as an error, exactly as the reference does
 * (presolve/gpu_presolve.hpp:25-26). */
enum {
  GPP_OK = 0,
  GPP_ERR_CUDA = 1,          /* maps to std::runtime_error("context: cudaGetErrorString") */
  GPP_ERR_LENGTH = 2,        /* maps to std::length_error (offset overflow, offset.hpp:20-30) */
  GPP_ERR_INVALID = 3,       /* maps to std::invalid_argument (bad CSR / tolerance, folding.cu:79-81) */
  GPP_ERR_RUNTIME = 4,       /* other std::runtime_error */
  GPP_ERR_NO_DEVICE = 5      /* the CUDA extension cannot run: no device */
};

typedef struct gpp_csr {
  int32_t rows;
  int32_t cols;
  gpp_offset nnz;
  gpp_offset* rowPtr;
  int32_t* colVal;
  double* nzVal;
} gpp_csr;

typedef struct gpp_lp {
  gpp_csr A;
  gpp_csr AT;
  double* c;
  double* AL;
  double* AU;
  double* l;
  double* u;
  double obj_constant;
  gpp_offset AT_leading_slack;
  gpp_offset* AT_slack_after;
} gpp_lp;

/* Field order and defaults of PresolveParams (presolve_structs.hpp:28-158).
 * bools are uint8_t; the residual-bound-mode enum is a uint8_t. */
typedef struct gpp_params {
  int32_t max_iters;
  double max_time;
  uint8_t verbose;
  uint8_t record_postsolve_tape;
  uint8_t record_postsolve_tape_cpu;
  uint8_t enable_presolve;
  uint8_t enable_folding;
  double folding_tolerance;
  double feasibility_tol;
  double bound_tol;
  double zero_tol;
  double bound_strengthening_upper_relaxation_factor;
  int32_t bound_strengthening_max_rounds;
  int32_t bound_strengthening_max_bound_only_rounds;
  uint8_t bound_strengthening_preserve_free_zero_cost;
  int32_t doubleton_equations_max_fill_in_proxy;
  uint8_t doubleton_equations_scan;
  int32_t doubleton_equations_min_selected_per_batch;
  double doubleton_equations_min_selected_ratio;
  int32_t doubleton_equations_max_batch_rounds;
  double doubleton_equations_max_time;
  uint8_t enable_infeasible_and_fixed_variables;
  uint8_t enable_empty_rows;
  uint8_t enable_singleton_rows;
  uint8_t enable_infeasible_and_redundant_rows;
  uint8_t enable_bound_strengthening;
  uint8_t enable_parallel_rows;
  uint8_t enable_empty_columns;
  uint8_t enable_singleton_columns;
  uint8_t enable_doubleton_equations;
  uint8_t enable_dual_fix;
  int32_t dual_fix_max_nonzero_cost_col_degree;
  uint8_t enable_parallel_columns;
  double parallel_columns_max_abs_ratio;
  int32_t parallel_columns_scale_guard_max_group_size;
  int32_t parallel_columns_scale_guard_min_groups;
  /* The structure-specific startup rules (column domination, two-row
   * variable elimination, zero-cost product variables, the variable-pair
   * and absolute-value piecewise-linear reformulations) run as in the
   * reference. */
  uint8_t enable_structure_specific_rules;
  uint8_t enable_two_row_variable_elimination;
  int32_t two_row_variable_elimination_max_row_nnz;
  double two_row_variable_elimination_safety_tol;
  int32_t two_row_variable_elimination_min_candidates;
  double two_row_variable_elimination_min_candidate_ratio;
  uint8_t enable_zero_cost_product_variables;
  int32_t zero_cost_product_variables_min_candidates;
  double zero_cost_product_variables_min_candidate_ratio;
  uint8_t enable_piecewise_linear_reformulation_variable_pair;
  int32_t piecewise_linear_reformulation_variable_pair_epigraph_probe_pairs;
  int32_t piecewise_linear_reformulation_variable_pair_epigraph_min_pairs;
  double piecewise_linear_reformulation_variable_pair_epigraph_min_potential_gain;
  double piecewise_linear_reformulation_variable_pair_epigraph_min_actual_gain;
  int32_t piecewise_linear_reformulation_variable_pair_epigraph_max_tail_cols;
  int32_t piecewise_linear_reformulation_variable_pair_epigraph_max_quotient_terms_per_row;
  int32_t piecewise_linear_reformulation_variable_pair_shifted_antipodal_probe_pairs;
  int32_t piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs;
  double piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_potential_gain;
  double piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_actual_gain;
  int32_t piecewise_linear_reformulation_variable_pair_shifted_antipodal_max_quotient_terms_per_row;
  uint8_t enable_column_domination;
  int32_t column_domination_probe_rows;
  int32_t column_domination_probe_cols;
  int32_t column_domination_probe_nnz;
  int32_t column_domination_min_fixed_cols;
  double column_domination_min_candidate_ratio;
  uint8_t enable_piecewise_linear_reformulation_absolute_value;
  uint8_t piecewise_linear_reformulation_absolute_value_residual_bound_mode;
  double piecewise_linear_reformulation_absolute_value_residual_bound_as_free_min;
  uint8_t enable_redundant_variable_bounds;
  uint8_t enable_startup;
  int64_t bound_strengthening_bound_only_nnz_round_budget;
} gpp_params;

/* piecewise_linear_reformulation_absolute_value_residual_bound_mode values
 * (PiecewiseLinearReformulationAbsoluteValueResidualBoundMode,
 * presolve_structs.hpp:15-26). */
#define GPP_RESIDUAL_PRESERVE_FINITE 0
#define GPP_RESIDUAL_STRICT_FREE_ONLY 1
#define GPP_RESIDUAL_LEGACY_WIDE_AS_FREE 2

/* Reference defaults (presolve_structs.hpp:28-158). */
GPP_API void gpp_default_params(gpp_params* params);

/* Opaque GPU-resident postsolve record (PresolveRecordGpu's device state,
 * presolve_structs.hpp:338-368).  Owned by the summary. */
typedef struct gpp_record gpp_record;

/* GpuPresolveSummary (presolve/gpu_presolve.hpp:14-30) merged with the
 * pipeline fields of FoldingPipelineSummary (folding/folding_structs.hpp:94-109). */
typedef struct gpp_summary {
  int32_t original_rows;
  int32_t original_cols;
  int32_t reduced_rows;
  int32_t reduced_cols;
  gpp_offset reduced_nnz;
  int32_t iterations;
  uint8_t stopped_at_iteration_limit;
  uint8_t has_change;
  uint8_t has_infeasible;
  uint8_t has_unbounded;
  uint8_t presolve_enabled;
  uint8_t folding_applied;
  uint8_t owns_reduced_lp;
  double elapsed_seconds;          /* presolve core wall time */
  double preprocessing_seconds;    /* whole preprocess() wall time */
  double obj_constant_delta;
  gpp_lp reduced_lp;               /* device arrays; borrowed from the input when !owns_reduced_lp */
  gpp_record* record;
  int32_t folded_rows;             /* sizes of the folded model (the original sizes when not folded) */
  int32_t folded_cols;
} gpp_summary;

/* ---- Plain pipeline: preprocess / postprocess / free_summary ------------- */

/* gpu_preprocessor::preprocess (cpp/include/gpu_preprocessor/gpu_preprocessor.hpp:22-24),
 * i.e. folding::run_gpu_presolve_with_folding(lp, params, true, true)
 * (folding/folding.hpp:48-51).  `lp` is caller-owned device data and is never
 * written.  The input must provide both A and AT = A^T in CSR form. */
GPP_API int gpp_preprocess(const gpp_lp* lp, const gpp_params* params, gpp_summary* out);

/* presolve::run_gpu_presolve_with_reduced_lp (presolve/gpu_presolve.hpp:35-36):
 * presolve only, reduced LP kept.  keep_reduced_lp = 0 gives
 * run_gpu_presolve_with_record (gpu_presolve.hpp:32-33). */
GPP_API int gpp_run_presolve(const gpp_lp* lp, const gpp_params* params, int keep_reduced_lp,
                     gpp_summary* out);

/* gpu_preprocessor::postprocess (gpu_preprocessor.hpp:30-33) /
 * folding::postsolve_and_unfold_to_host (folding/folding.hpp:53-57).
 * x_red (reduced_cols), y_red (reduced_rows), z_red (reduced_cols) are
 * caller-owned device arrays in reduced order; any may be NULL.  x_out (n0),
 * y_out (m0), z_out (n0) are HOST arrays in original order.  Dual convention
 * c - A^T y - z = 0.  `original` must be the LP given to preprocess. */
GPP_API int gpp_postprocess(const double* x_red, const double* y_red, const double* z_red,
                    const gpp_summary* summary, const gpp_lp* original,
                    double* x_out, double* y_out, double* z_out);

/* presolve::postsolve_gpu (presolve/gpu_postsolve.hpp:20-31): same as
 * gpp_postprocess but x_org/y_org/z_org are DEVICE arrays (n0, m0, n0) that
 * the caller owns.  `original` may be NULL (primal-only recovery, no dual
 * projection). */
GPP_API int gpp_postsolve_device(const double* x_red, const double* y_red, const double* z_red,
                         const gpp_summary* summary, const gpp_lp* original,
                         double* x_org, double* y_org, double* z_org);

/* postsolve_gpu with its original_l argument (gpu_postsolve.hpp:26-31):
 * original_l (DEVICE, n0 entries, may be NULL) bounds the absolute-value
 * reformulation's max slacks below; when NULL, original->l is used (0 when
 * `original` is NULL too).  gpp_postsolve_device is this with NULL. */
GPP_API int gpp_postsolve_device_lower(const double* x_red, const double* y_red, const double* z_red,
                                       const gpp_summary* summary, const gpp_lp* original,
                                       const double* original_l, double* x_org, double* y_org, double* z_org);

/* gpu_preprocessor::free_summary (gpu_preprocessor.hpp:35-39) /
 * presolve::free_gpu_presolve_reduced_lp (gpu_presolve.hpp:38).
 * Idempotent: a second call is a no-op. */
GPP_API void gpp_free_summary(gpp_summary* summary);

/* Export of the recovery maps (the reference's export_recovery_record,
 * presolve/device_recovery.hpp:84).  Host arrays of length reduced_rows and
 * reduced_cols receive the original index of every kept row / column. */
GPP_API int gpp_export_maps(const gpp_summary* summary, int32_t* row_red2org, int32_t* col_red2org);

/* Size of the postsolve tape held by the record (records, indices, values,
 * fixed-value entries). */
GPP_API int gpp_tape_sizes(const gpp_summary* summary, int64_t* records, int64_t* indices,
                   int64_t* values, int64_t* fixed);

/* Copies the tape to host arrays (types[records], index_starts[records+1],
 * value_starts[records+1], indices[indices], vals[values], fixed_idx[fixed],
 * fixed_val[fixed]); any pointer may be NULL. */
GPP_API int gpp_export_tape(const gpp_summary* summary, int32_t* types, int64_t* index_starts,
                    int64_t* value_starts, int32_t* indices, double* vals,
                    int32_t* fixed_idx, double* fixed_val);

/* ---- Piecewise-linear primal recoveries ---------------------------------- */

/* Layout an absolute-value reformulation matched: the reference's recovery
 * `pattern` strings (rule_piecewise_linear_reformulation_absolute_value.cu:
 * "l1_split_3row" :1998, "graph_l1_substitution" :2235,
 * "outer_pair_linked_l1" :2683). */
#define GPP_ABS_L1_SPLIT 1
#define GPP_ABS_GRAPH_L1 2
#define GPP_ABS_OUTER_PAIR 3

/* One absolute-value primal recovery step
 * (PiecewiseLinearReformulationAbsoluteValuePrimalRecoveryStep,
 * presolve_structs.hpp:207-236) as HOST arrays of original column ids.
 * Applied as: splits (t, e) <- (t + e, (t - e) / rho); outer pairs
 * free <- bound; linked slacks slack <- factor * t; max-slack group g
 * (entries [max_starts[g], max_starts[g + 1])) slack <- max(l_slack,
 * max factor * t). */
typedef struct gpp_absolute_value_recovery {
  int32_t pattern;
  int32_t split_count;
  const int32_t* split_t;
  const int32_t* split_e;
  const double* split_rho;
  int32_t pair_count;
  const int32_t* pair_bound;
  const int32_t* pair_free;
  int32_t linked_count;
  const int32_t* linked_slack;
  const int32_t* linked_t;
  const double* linked_factor;
  int32_t max_group_count;
  const int32_t* max_slack;
  const int32_t* max_starts;    /* max_group_count + 1 entries */
  const int32_t* max_t;
  const double* max_factor;
} gpp_absolute_value_recovery;

/* The record's primal-recovery checkpoints (primal_recovery_timeline,
 * presolve_structs.hpp:256-266, 362).  *count is always written; kinds
 * (0 = absolute value, 1 = variable pair), payloads (index of the recovery of that kind) and
 * tape_positions (records replayed before the recovery is applied), when not
 * NULL, receive *count entries. */
GPP_API int gpp_recovery_checkpoints(const gpp_summary* summary, int32_t* count, int32_t* kinds,
                                     int32_t* payloads, int64_t* tape_positions);

/* Sizes of absolute-value recovery `index`: sizes[0] pattern, [1] splits,
 * [2] outer pairs, [3] linked slacks, [4] max-slack groups, [5] max-slack
 * entries. */
GPP_API int gpp_absolute_value_sizes(const gpp_summary* summary, int32_t index, int32_t sizes[6]);

/* Copies absolute-value recovery `index` to HOST arrays sized by
 * gpp_absolute_value_sizes (max_starts: groups + 1); any pointer may be NULL. */
GPP_API int gpp_export_absolute_value(const gpp_summary* summary, int32_t index, int32_t* split_t,
                                      int32_t* split_e, double* split_rho, int32_t* pair_bound,
                                      int32_t* pair_free, int32_t* linked_slack, int32_t* linked_t,
                                      double* linked_factor, int32_t* max_slack, int32_t* max_starts,
                                      int32_t* max_t, double* max_factor);

/* Size (pairs) of variable-pair recovery `index`
 * (PiecewiseLinearReformulationVariablePairRecoveryStep, presolve_structs.hpp:243-250). */
GPP_API int gpp_variable_pair_size(const gpp_summary* summary, int32_t index, int32_t* count);

/* Copies variable-pair recovery `index` to HOST arrays of *count entries
 * (original column ids; x[plus] = plus_shift + x[root_plus], likewise for
 * minus); any pointer may be NULL. */
GPP_API int gpp_export_variable_pair(const gpp_summary* summary, int32_t index, int32_t* plus_cols,
                                     int32_t* minus_cols, int32_t* root_plus_cols, int32_t* root_minus_cols,
                                     double* plus_shift, double* minus_shift);

/* postsolve_restore_piecewise_linear_reformulation_absolute_value_gpu
 * (presolve/gpu_postsolve.hpp:15-18): applies `count` steps to the DEVICE
 * vector x_org, the last step first.  original_l (DEVICE, may be NULL) gives
 * the max slacks' lower bounds (0 when NULL or not finite).  Column ids must
 * be below the length of x_org; they are not checked against it. */
GPP_API int gpp_restore_absolute_value(double* x_org, const gpp_absolute_value_recovery* steps,
                                       int32_t count, const double* original_l);

/* folding::copy_map_to_host (folding/folding.hpp:22): the 1-based colour of
 * every original row / column and the unfold scales 1/|colour|, as HOST
 * arrays (m0, n0, m0, n0; any may be NULL).  Returns GPP_OK with nothing
 * written when folding did not apply (summary->folding_applied == 0). */
GPP_API int gpp_export_folding_map(const gpp_summary* summary, int32_t* row_color, int32_t* col_color,
                                   double* row_scale, double* col_scale);

/* folding::run_folding / free_folded_lp (folding/folding.hpp:16-20): colour
 * refinement and the quotient LP of `lp` alone, without presolve.  When
 * folding applies, `folded_lp` is a device model owned by the run
 * (owns_folded_lp = 1) and the four map arrays are device arrays of the
 * original sizes (1-based colours, unfold scales 1/|colour|); otherwise
 * `applied` = 0, folded sizes equal the original ones, `folded_lp` is zero
 * and the map pointers are NULL, as the reference's summary is.  A negative
 * or non-finite tolerance gives GPP_ERR_INVALID.
 * gpp_free_folding_run releases everything the run owns; calling it twice
 * is safe. */
typedef struct gpp_folding_run {
  uint8_t applied;
  int32_t original_rows, original_cols, folded_rows, folded_cols;
  double seconds;
  gpp_lp folded_lp;
  uint8_t owns_folded_lp;
  int32_t* row_color_id;
  int32_t* col_color_id;
  double* row_scale;
  double* col_scale;
  void* handle;
} gpp_folding_run;
GPP_API int gpp_run_folding(const gpp_lp* lp, double tolerance, gpp_folding_run* out);
GPP_API void gpp_free_folding_run(gpp_folding_run* run);
/* gpp_export_folding_map and gpp_unfold_solution for the map of a
 * gpp_run_folding result (same outputs; nothing written / an invalid
 * argument when folding did not apply). */
GPP_API int gpp_folding_run_export_map(const gpp_folding_run* run, int32_t* row_color, int32_t* col_color,
                                       double* row_scale, double* col_scale);
GPP_API int gpp_folding_run_unfold(const gpp_folding_run* run, const double* x_folded, const double* y_folded,
                                   const double* z_folded, double* x_out, double* y_out, double* z_out);

/* folding::unfold_solution_device_to_host (folding/folding.hpp:40-44): map a
 * solution of the folded model (DEVICE arrays of folded_cols, folded_rows,
 * folded_cols entries; any may be NULL) to the original model on the HOST:
 * x_j = x_f[C(j)], y_i = y_f[R(i)] / |R(i)|, z_j = z_f[C(j)] / |C(j)|. */
GPP_API int gpp_unfold_solution(const gpp_summary* summary, const double* x_folded, const double* y_folded,
                                const double* z_folded, double* x_out, double* y_out, double* z_out);

/* ---- Batched form --------------------------------------------------------- */

/* Presolves `count` independent LPs (lps[k] -> out[k]), each exactly as
 * gpp_preprocess would: the same rules, the same results.  The LPs are spread
 * over `workers` host threads of the library (workers <= 0: 8), each with its
 * own stream on the current device, largest LP first, so that many small LPs
 * keep the GPU busy while each one waits on its own host round-trips.  The
 * threads are created on first use and kept until exit.  status[k] (may be
 * NULL) receives LP k's status; the return value is GPP_OK or the first
 * failing LP's status, with gpp_last_error naming that LP.  Free every out[k]
 * with gpp_free_summary, whether or not the batch succeeded.  The reference has
 * no batched entry point; this is the batched form of its plain path. */
GPP_API int gpp_preprocess_batch(const gpp_lp* lps, int32_t count, const gpp_params* params, int32_t workers,
                                 gpp_summary* out, int32_t* status);

/* gpp_postprocess for each LP of a batch, on the same worker threads:
 * x_red[k], y_red[k], z_red[k] are LP k's reduced solution (device; the
 * arrays of pointers, and any entry, may be NULL), x_out[k], y_out[k],
 * z_out[k] its host outputs in original order. */
GPP_API int gpp_postprocess_batch(const double* const* x_red, const double* const* y_red,
                                  const double* const* z_red, const gpp_summary* summaries,
                                  const gpp_lp* originals, int32_t count, int32_t workers,
                                  double* const* x_out, double* const* y_out, double* const* z_out,
                                  int32_t* status);

/* Chooses the worker count for a batch: times gpp_preprocess_batch on a
 * sample of up to 32 of the LPs (every k-th by size) with 1, 2, 4, ... up to
 * max_workers threads and writes the count of the best throughput (a larger
 * count must win by 5%).  `rates` (may be NULL; one entry per count tried,
 * floor(log2(max_workers)) + 1 of them) receives the sampled LPs/s. */
GPP_API int gpp_batch_autotune(const gpp_lp* lps, int32_t count, const gpp_params* params, int32_t max_workers,
                               int32_t* best_workers, double* rates);

/* ---- Host I/O: MPS input, reduced-LP export -------------------------------- */

/* A continuous LP read from an MPS file (the reference's mps_reader::read_mps,
 * cpp/mps_reader/include/mps_reader/mpsreader.hpp:13-18, same arrays for the
 * same file): free format, or fixed columns when free parsing fails; ROWS,
 * COLUMNS (integer markers read as bounds only), RHS (an RHS on the objective
 * row is the negated objective constant), RANGES, BOUNDS (FR MI PL BV LO UP FX
 * LI UI), OBJSENSE MIN.  Duplicate coefficients are summed.  Errors:
 * GPP_ERR_INVALID with the parser's message. */
typedef struct gpp_mps_model gpp_mps_model;
GPP_API int gpp_mps_read(const char* path, gpp_mps_model** out);
GPP_API int gpp_mps_read_string(const char* text, gpp_mps_model** out);
/* Sizes, objective constant and model name (NUL-terminated, truncated to
 * name_len); any pointer may be NULL. */
GPP_API int gpp_mps_info(const gpp_mps_model* model, int32_t* rows, int32_t* cols, int64_t* nnz,
                         double* obj_constant, char* name, size_t name_len);
/* Host copies: CSR (row_ptr[rows+1], col_idx, csr_val), CSC (col_ptr[cols+1],
 * row_idx, csc_val; columns in file order, rows ascending), c[cols],
 * AL/AU[rows], l/u[cols]; any pointer may be NULL. */
GPP_API int gpp_mps_arrays(const gpp_mps_model* model, int64_t* row_ptr, int32_t* col_idx, double* csr_val,
                           int64_t* col_ptr, int32_t* row_idx, double* csc_val, double* c, double* AL, double* AU,
                           double* l, double* u);
GPP_API void gpp_mps_free(gpp_mps_model* model);
/* The model on the current device as a gpp_lp with A and AT = A^T (the
 * reference's tools upload_lp, cpp/tools/gpu_preprocessor_tool_common.hpp:
 * 108-141); the arrays are cudaMalloc'd and released by gpp_lp_free. */
GPP_API int gpp_mps_upload(const gpp_mps_model* model, gpp_lp* out);
GPP_API void gpp_lp_free(gpp_lp* lp);

/* An LP in host memory: A as CSR (row_ptr[rows+1], col_idx[nnz], val[nnz])
 * and the vectors c/l/u[cols], AL/AU[rows].  No transpose. */
typedef struct gpp_host_lp {
  int32_t rows;
  int32_t cols;
  gpp_offset nnz;
  const gpp_offset* row_ptr;
  const int32_t* col_idx;
  const double* val;
  const double* c;
  const double* AL;
  const double* AU;
  const double* l;
  const double* u;
  double obj_constant;
} gpp_host_lp;
/* Loads a host LP into device arrays the caller allocated on the current
 * device (dev->A.rowPtr[rows+1], A.colVal/A.nzVal[nnz], AT.rowPtr[cols+1],
 * AT.colVal/AT.nzVal[nnz], c/l/u[cols], AL/AU[rows]) and builds AT = A^T on
 * the GPU, each column listing its rows in ascending order (the CSC that
 * upload_lp copies from the host, cpp/tools/gpu_preprocessor_tool_common.hpp:
 * 108-141).  Only A and the vectors cross PCIe: the transpose is built from
 * the uploaded A while the vectors are still being copied.  Sets dev's sizes
 * and obj_constant; the call returns when the device arrays are complete.
 * Host arrays may be pageable or page-locked (page-locked copies run
 * asynchronously at full bus speed).  GPP_ERR_INVALID for a structurally
 * invalid A (row pointers not starting at 0, decreasing or not ending at nnz;
 * a column index outside [0, cols)), checked on the device before the
 * transpose reads it. */
GPP_API int gpp_lp_from_host(const gpp_host_lp* host, gpp_lp* dev);

/* Writes the reduced LP of a summary to `out_dir` in the reference's export
 * format (cpp/tools/gpu_preprocessor_export_reduced.cpp:17-64, format
 * gpu_preprocessor_reduced_lp_v1): meta.txt and the raw little-endian arrays
 * A_rowPtr_i32, A_colVal_i32, A_nzVal_f64, c_f64, l_f64, u_f64, AL_f64,
 * AU_f64 (.bin).  meta.txt has the reference's keys except folding_seconds,
 * which this engine does not time separately. */
GPP_API int gpp_export_reduced(const gpp_summary* summary, const char* out_dir, const char* model_name);

/* Solver handoff of the reduced LP (the reference's HPR-LP adapter,
 * solver_interface/adapters/gpu.cpp:354-400 and :466-500).
 *
 * gpp_reduced_to_device copies the reduced LP, device to device, into new
 * arrays on the current device that the caller owns and releases with
 * gpp_lp_free: A, its stable transpose AT (rows of AT list the rows of A in
 * ascending order, as build_stable_device_transpose makes them), c, AL, AU,
 * l, u and the objective constant.  It fails with GPP_ERR_INVALID when the
 * reduced LP is empty (no rows, columns or nonzeros), where the reference's
 * adapter reports that preprocessing failed.
 *
 * gpp_reduced_to_host copies the same arrays to host buffers of the sizes in
 * the summary (row_ptr: reduced_rows + 1; col_idx, val: reduced_nnz; c, l, u:
 * reduced_cols; AL, AU: reduced_rows); any pointer may be NULL to skip that
 * array. */
GPP_API int gpp_reduced_to_device(const gpp_summary* summary, gpp_lp* out);
GPP_API int gpp_reduced_to_host(const gpp_summary* summary, gpp_offset* row_ptr, int32_t* col_idx, double* val,
                                double* c, double* AL, double* AU, double* l, double* u, double* obj_constant);

/* ---- Learned round schedule -------------------------------------------------
 * The plain phase machine (Cleanup, Propagation, Aggregation, Parallel) runs
 * one phase per round.  A schedule model may, per round, skip any of six gated
 * rules (singleton columns, bound strengthening, redundant rows + dual fix,
 * doubleton equations, parallel rows, parallel columns) and stop presolve.
 * The model is a small FP32 MLP with GPP_SCHEDULE_FEATURES inputs, two hidden
 * layers of GPP_SCHEDULE_HIDDEN units and GPP_SCHEDULE_OUTPUTS logits (one per
 * gated rule, "the rule will change the model this round", then "stop").
 * The reference has no counterpart; its plain loop stays the default here. */
#define GPP_SCHEDULE_FEATURES 32
#define GPP_SCHEDULE_HIDDEN 64
#define GPP_SCHEDULE_OUTPUTS 7
/* W1[24][64], b1[64], W2[64][64], b2[64], W3[64][7], b3[7], row-major. */
#define GPP_SCHEDULE_PARAMS (32 * 64 + 64 + 64 * 64 + 64 + 64 * 7 + 7)

/* gpp_preprocess that also records every round: features[r * 24 + i],
 * round_info[4 r ..] = phase (0 Cleanup, 1 Propagation, 2 Aggregation,
 * 3 Parallel), iteration, gated rules that ran (bit mask), gated rules that
 * changed the model (bit mask); round_nnz[2 r ..] = live nnz before and after
 * the round.  At most max_rounds are written; *rounds gets the count.  The
 * presolve result is the plain one. */
GPP_API int gpp_preprocess_traced(const gpp_lp* lp, const gpp_params* params, gpp_summary* out, float* features,
                                  int32_t* round_info, int64_t* round_nnz, int32_t max_rounds, int32_t* rounds);

typedef struct gpp_schedule_model gpp_schedule_model;
/* A model from GPP_SCHEDULE_PARAMS host floats.  Per round it skips gated rule
 * g when sigmoid(logit g) < skip_below and stops when sigmoid(stop logit) >
 * stop_above (skip_below = 0 keeps every rule; stop_above >= 1 never stops).
 * One model may be used by one host thread at a time. */
GPP_API int gpp_schedule_model_create(const float* params, double skip_below, double stop_above,
                                      gpp_schedule_model** out);
/* The same with one skip threshold per gated rule (GPP_SCHEDULE_GATED_RULES
 * values, in the order singleton columns, bound strengthening, redundant rows
 * + dual fix, doubleton equations, parallel rows, parallel columns). */
#define GPP_SCHEDULE_GATED_RULES 6
GPP_API int gpp_schedule_model_create_per_rule(const float* params, const double* skip_below, double stop_above,
                                               gpp_schedule_model** out);
GPP_API void gpp_schedule_model_free(gpp_schedule_model* model);
/* gpp_preprocess with the rounds scheduled by `model`. */
GPP_API int gpp_preprocess_scheduled(const gpp_lp* lp, const gpp_params* params, gpp_schedule_model* model,
                                     gpp_summary* out);

/* Training and inference of the schedule MLP on the GPU (host arrays in and
 * out).  X is n x 32, Y and M (labels and 0/1 masks) are n x 7; the loss is
 * the mean over samples of the masked binary cross-entropy of the logits.
 * gpp_mlp_train runs `epochs` epochs of Adam (minibatches of `batch`, order
 * shuffled by `seed`) from and into `params`; loss_per_epoch may be NULL. */
GPP_API int gpp_mlp_train(float* params, const float* X, const float* Y, const float* M, int64_t n, int32_t epochs,
                          int32_t batch, float lr, uint64_t seed, float* loss_per_epoch);
GPP_API int gpp_mlp_forward(const float* params, const float* X, int64_t n, float* probs);
GPP_API int gpp_mlp_gradients(const float* params, const float* X, const float* Y, const float* M, int64_t n,
                              float* grads, float* loss);

/* ---- Kernel-level entry points (rule / kernel parity tests) -------------- */

/* compute_row_activity_summary (presolve/gpu_presolve_kernels.hpp:76-86):
 * per row finite min/max activity and counts of -inf/+inf contributions,
 * entries with |a| <= zero_tol skipped, optional keep masks (NULL = all kept)
 * and optional live degrees used for the short/medium/long row split.  All
 * pointers are device pointers; runs on the legacy default stream. */
GPP_API int gpp_row_activity_summary(const gpp_csr* A, const double* l, const double* u,
                             double zero_tol, const uint8_t* keep_row,
                             const uint8_t* keep_col, const int32_t* live_degrees,
                             double* min_fin, double* max_fin,
                             int32_t* min_inf, int32_t* max_inf);

/* refresh_live_stats (presolve/gpu_presolve_kernels.hpp:45-56) for one side:
 * live degree, empty / singleton flags, singleton support index and value of
 * every row of `M` under keep_outer (rows) and keep_inner (columns), plus the
 * live nonzero total (device u64, may be NULL). */
GPP_API int gpp_live_stats(const gpp_csr* M, const uint8_t* keep_outer, const uint8_t* keep_inner,
                   int32_t* degree, uint8_t* empty, uint8_t* singleton,
                   int32_t* support, double* coefficient, unsigned long long* total);

/* compute_col_max_abs (gpu_presolve_kernels.hpp:88-89): max |a| per row of AT
 * over kept rows of A. */
GPP_API int gpp_col_max_abs(const gpp_csr* AT, const uint8_t* keep_row, double* col_max_abs);

/* Stable CSR compaction by row/column keep masks followed by the transpose
 * (apply_plan_to_working_lp's compact_csr_by_masks_gpu + transpose_csr64,
 * cpp/src/presolve/gpu_presolve.cu:1793-1930, transpose64.cu:54-117).
 * Outputs are newly allocated device arrays owned by the caller (free with
 * gpp_device_free). */
GPP_API int gpp_compact_and_transpose(const gpp_csr* A, const uint8_t* keep_row, const uint8_t* keep_col,
                              gpp_csr* A_out, gpp_csr* AT_out);

/* Parallel-row hashes (rule_parallel_rows.cu:132-343): FNV-1a fold of the
 * pivot-normalised live pattern of every row, mode 0 sequential, 1 XOR
 * aggregate. */
GPP_API int gpp_parallel_row_hashes(const gpp_csr* A, const uint8_t* keep_row, const uint8_t* keep_col,
                            int mode, uint64_t* hashes);

/* Stable sort of n (uint64 key, int32 value) device pairs by key, in place:
 * the engine's radix sort that replaces the reference's thrust::sort of
 * (hash, id) tuples (rule_parallel_rows.cu:742-770). */
GPP_API int gpp_sort_pairs(uint64_t* keys, int32_t* values, int64_t n);

/* The same stable sort of n (uint64 key, int32 value) device pairs, for
 * callers that cannot allocate device memory when they call it: an LP solver
 * that hands the whole device to its own arena allocator, or a host
 * application that was promised a fixed device footprint, cannot let this
 * library call cudaMalloc or grow a memory pool on its behalf.  This entry
 * point has no counterpart in the reference.
 *
 * Its scratch is one fixed device array inside the library, sized for
 * GPP_SORT_STATIC_MAX_PAIRS pairs (about 12.5 MiB); a larger n returns
 * GPP_ERR_LENGTH without touching the data.  A call launches kernels on
 * `stream` (a cudaStream_t; NULL for the legacy default stream) and returns
 * without synchronizing; it calls no cudaMalloc, cudaFree or allocating
 * library routine.  The first call on each device (any n, 0 included) loads
 * the library's device code on that device, which places the fixed array in
 * device memory, and looks up the array's device address with that device
 * current: make that first call before an arena allocator takes the device's
 * memory and before any stream capture.  The address is kept for the life of
 * the process, so do not use this entry point on a device after
 * cudaDeviceReset.  Every call shares the one array, so calls whose work
 * overlaps on the GPU race and give wrong results: order them on one stream
 * or synchronize between them.  Output equals gpp_sort_pairs'. */
#define GPP_SORT_STATIC_MAX_PAIRS (1 << 20)
GPP_API int gpp_sort_pairs_static(uint64_t* keys, int32_t* values, int64_t n, void* stream);

/* Device allocation of `bytes` bytes with cudaMalloc (the C++ layer's
 * postsolve_gpu returns such arrays, as the reference's does,
 * cpp/src/presolve/gpu_postsolve.cu:545-556).  Release with gpp_device_free or
 * cudaFree.  bytes = 0 gives NULL. */
GPP_API int gpp_device_alloc(void** device_ptr, size_t bytes);
GPP_API void gpp_device_free(void* device_ptr);

/* Test hook for failure handling: the device allocation made `after`
 * allocations from now (0 = the next one, counted over all threads) by any
 * engine entry point returns cudaErrorMemoryAllocation instead of memory,
 * exactly once; `after` < 0 disarms it.  The failing call returns
 * GPP_ERR_CUDA with its message and releases what it had allocated; the
 * device is not touched, so later calls run normally. */
GPP_API void gpp_inject_alloc_failure(int64_t after);

/* Last error message of the calling thread ("" when none). */
GPP_API const char* gpp_last_error(void);

/* Per-kernel timing for the benchmark's roofline report.  While enabled,
 * every launch on the calling thread is bracketed by CUDA events on its
 * stream; gpp_profile_read aggregates by kernel name (launches, total ms,
 * algorithmic bytes the launch was charged) and returns the number of kernel
 * names, filling entry `index` when it exists.  Enabling clears old records. */
GPP_API void gpp_profile_enable(int enable);
GPP_API int gpp_profile_read(int index, char* name, size_t name_len, int64_t* launches, double* ms,
                             double* bytes);

/* Number of CUDA kernels this library launched on the calling thread since
 * the last reset (used by the benchmark to report its launch count). */
GPP_API uint64_t gpp_kernel_launches(int reset);

/* Number of times the library waited on its stream from the calling thread
 * (to read a count, a flag or a size back) since the last reset: each wait
 * leaves the GPU idle until the host launches again. */
GPP_API uint64_t gpp_host_syncs(int reset);

#ifdef __cplusplus
}
#endif

#endif /* GPP_H_ */
