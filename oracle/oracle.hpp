// Oracle: a single-threaded CPU restatement of GPU-Preprocessor's plain
// presolve + postsolve path.  TEST INFRASTRUCTURE ONLY: it is the checker for
// the CUDA engine and is never linked into, called by, or shipped with it.
//
// Each routine cites the reference file:line it restates (paths relative to
// the reference's project root).  Floating-point reductions follow the
// reference's association order where the reference is deterministic (row
// activity buckets, CUB block/warp reduction trees, long-double objective
// sums); where the reference uses order-dependent atomicAdd (row shifts,
// fixed-variable error budgets) the oracle uses ascending column order, the
// same order the CUDA engine commits to.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../include/gpp.h"

namespace oracle {

struct Csr {
  int rows = 0, cols = 0;
  std::vector<int> ptr{0};
  std::vector<int> idx;
  std::vector<double> val;
  int nnz() const { return ptr.empty() ? 0 : ptr.back(); }
};

Csr transpose(const Csr& a);

struct Lp {
  Csr A, AT;
  std::vector<double> c, AL, AU, l, u;
  double obj = 0.0;
  int m() const { return A.rows; }
  int n() const { return A.cols; }
};

// Chronological postsolve tape (same record vocabulary as the reference,
// presolve_structs.hpp:268-282).
struct Tape {
  std::vector<int> types;
  std::vector<int64_t> is{0}, vs{0};
  std::vector<int> idx;
  std::vector<double> val;
  int64_t count() const { return int64_t(types.size()); }
  void add(int type, const std::vector<int>& i, const std::vector<double>& v) {
    types.push_back(type);
    idx.insert(idx.end(), i.begin(), i.end());
    val.insert(val.end(), v.begin(), v.end());
    is.push_back(int64_t(idx.size()));
    vs.push_back(int64_t(val.size()));
  }
  void append(const Tape& t);
};

enum RecordType {
  FixedVariable = 0, InfiniteBoundDualFix = 1, SingletonColumnSubstitution = 2,
  ParallelColumn = 3, ParallelRow = 4, DeletedRow = 5, RowLowerBoundChange = 8,
  RowUpperBoundChange = 9, RowDualShift = 10, VariableBoundChange = 11,
  RowImpliedBoundChange = 12, DoubletonEquation = 13, FmeCol = 14
};

struct Stats {
  std::vector<int> row_nnz, col_nnz, srow_col, scol_row;
  std::vector<uint8_t> empty_row, singleton_row, empty_col, singleton_col;
  std::vector<double> srow_val, scol_val;
  int64_t live_nnz = 0;
};

struct Plan {
  std::vector<uint8_t> keep_row, keep_col;
  std::vector<double> c, l, u, AL, AU;
  double obj_delta = 0.0;
  bool has_change = false, has_row_action = false, has_col_action = false;
  bool has_redundant_row_deletion = false, has_row_deletion = false;
  bool has_infeasible = false, has_unbounded = false;
  const std::vector<uint8_t>* rule_entry_keep_col = nullptr;
  const std::vector<double>* ref_l = nullptr;
  const std::vector<double>* ref_u = nullptr;
  bool has_new_A = false;
  Csr new_A;
  Tape tape;  // local indices until captured
};

struct Record {
  int m0 = 0, n0 = 0;
  std::vector<int> rows, cols;       // current index -> original index
  std::vector<int> fixed_idx;
  std::vector<double> fixed_val;
  Tape tape;                          // original indices
};

struct Result {
  gpp_summary summary{};
  Lp reduced;
  Record record;
  std::vector<std::string> trace;     // phase / rule trace (schedule tests)
};

// --- kernel-level restatements -------------------------------------------
void row_activity_summary(const Csr& A, const std::vector<double>& l, const std::vector<double>& u,
                          double zero_tol, const uint8_t* keep_row, const uint8_t* keep_col,
                          const int* live_degrees, double* min_fin, double* max_fin,
                          int* min_inf, int* max_inf);
void row_activity_impl(const Csr& A, const std::vector<double>& l, const std::vector<double>& u,
                       double zero_tol, const uint8_t* keep_row, const uint8_t* keep_col,
                       const int* live_degrees, double* min_fin, double* max_fin, int* min_inf, int* max_inf,
                       bool plain);
void row_plain_minmax(const Csr& A, const std::vector<double>& l, const std::vector<double>& u,
                      const uint8_t* keep_row, const uint8_t* keep_col, const int* live_degrees,
                      double* row_min, double* row_max);
void live_stats(const Csr& M, const uint8_t* keep_outer, const uint8_t* keep_inner, int* degree,
                uint8_t* empty, uint8_t* singleton, int* support, double* coefficient,
                int64_t* total);
void col_max_abs(const Csr& AT, const uint8_t* keep_row, double* out);
uint64_t row_hash(const Csr& A, int row, const uint8_t* keep_col, int mode);
uint64_t row_hash_tol(const Csr& A, int row, const uint8_t* keep_col, int mode, double tol);
uint64_t col_hash(const Csr& AT, int col, const uint8_t* keep_row, double tol);

// --- folding (oracle_folding.cpp) -----------------------------------------
struct Fold {
  bool applied = false;
  int rows = 0, cols = 0;              // original sizes
  Lp folded;
  std::vector<int> row_color, col_color;     // 1-based colour per original row / column
  std::vector<double> row_scale, col_scale;  // 1 / colour size
};
Fold fold(const Lp& lp, double tol);

// --- pipeline -------------------------------------------------------------
Result presolve(const Lp& lp, const gpp_params& params);
void postsolve(const Result& r, const Lp& original, const double* x_red, const double* y_red,
               const double* z_red, double* x, double* y, double* z);

// Deterministic sum used for cleanup objective deltas (chunked fixed tree).
double det_sum(const std::vector<double>& v);

}  // namespace oracle
