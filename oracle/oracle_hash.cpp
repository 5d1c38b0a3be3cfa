// Oracle FNV-1a pattern hashes of the duplicate-detection rules.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <cmath>
#include <cstring>

#include "oracle.hpp"

namespace oracle {

namespace {
constexpr uint64_t kOffset = 0xcbf29ce484222325ULL, kPrime = 0x100000001b3ULL;
inline uint64_t mix(uint64_t h, uint64_t x) { return (h ^ x) * kPrime; }
inline uint64_t bits(double v) {
  uint64_t b;
  std::memcpy(&b, &v, 8);
  return b;
}
}  // namespace

uint64_t row_hash(const Csr& A, int row, const uint8_t* keep_col, int mode) {
  // _kernel_parallel_row_hashes (rule_parallel_rows.cu:141-190); mode 1 = XOR
  // aggregate, 0 = sequential fold.  Rows not kept are hashed by the caller.
  int first = -1, len = 0;
  for (int p = A.ptr[row]; p < A.ptr[row + 1]; ++p)
    if (!keep_col || keep_col[A.idx[p]]) { if (first < 0) first = p; ++len; }
  if (len == 0 || std::fabs(A.val[first]) <= 1e-10) return mix(kOffset, uint64_t(row));
  const double pivot = A.val[first];
  uint64_t h = mix(kOffset, uint64_t(len)), agg = 0;
  for (int p = first; p < A.ptr[row + 1]; ++p) {
    if (keep_col && !keep_col[A.idx[p]]) continue;
    const uint64_t b = bits(A.val[p] / pivot);
    if (mode) agg ^= mix(mix(kOffset, uint64_t(A.idx[p])), b);
    else h = mix(mix(h, uint64_t(A.idx[p])), b);
  }
  return mode ? mix(h, agg) : h;
}

uint64_t row_hash_tol(const Csr& A, int row, const uint8_t* keep_col, int mode, double tol) {
  int first = -1, len = 0;
  for (int p = A.ptr[row]; p < A.ptr[row + 1]; ++p)
    if (!keep_col || keep_col[A.idx[p]]) { if (first < 0) first = p; ++len; }
  if (len == 0 || std::fabs(A.val[first]) <= tol) return mix(kOffset, uint64_t(row));
  const double pivot = A.val[first];
  uint64_t h = mix(kOffset, uint64_t(len)), agg = 0;
  for (int p = first; p < A.ptr[row + 1]; ++p) {
    if (keep_col && !keep_col[A.idx[p]]) continue;
    const uint64_t b = bits(A.val[p] / pivot);
    if (mode) agg ^= mix(mix(kOffset, uint64_t(A.idx[p])), b);
    else h = mix(mix(h, uint64_t(A.idx[p])), b);
  }
  return mode ? mix(h, agg) : h;
}

uint64_t col_hash(const Csr& AT, int col, const uint8_t* keep_row, double tol) {
  // _kernel_parallel_column_hashes (rule_parallel_columns.cu:189-240).
  int len = 0;
  double pivot = 0.0;
  bool set = false;
  for (int p = AT.ptr[col]; p < AT.ptr[col + 1]; ++p)
    if (keep_row[AT.idx[p]] && std::fabs(AT.val[p]) > tol) { ++len; if (!set) { pivot = AT.val[p]; set = true; } }
  if (!set || len == 0) return mix(kOffset, uint64_t(col));
  uint64_t h = mix(kOffset, uint64_t(len));
  for (int p = AT.ptr[col]; p < AT.ptr[col + 1]; ++p)
    if (keep_row[AT.idx[p]] && std::fabs(AT.val[p]) > tol) h = mix(mix(h, uint64_t(AT.idx[p])), bits(AT.val[p] / pivot));
  return h;
}

}  // namespace oracle
