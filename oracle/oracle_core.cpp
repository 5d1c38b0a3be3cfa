// Oracle kernels: CPU restatements of the reference's per-row / per-column
// device kernels.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include "oracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>

namespace oracle {

Csr transpose(const Csr& a) {
  // cusparseCsr2cscEx2 semantics (transpose64.cu:54-117): rows of A^T list
  // the row indices of A in ascending order.
  Csr t;
  t.rows = a.cols;
  t.cols = a.rows;
  t.ptr.assign(size_t(a.cols) + 1, 0);
  for (int p = 0; p < a.nnz(); ++p) t.ptr[size_t(a.idx[p]) + 1]++;
  for (int j = 0; j < a.cols; ++j) t.ptr[j + 1] += t.ptr[j];
  t.idx.resize(size_t(a.nnz()));
  t.val.resize(size_t(a.nnz()));
  std::vector<int> next(t.ptr.begin(), t.ptr.end() - 1);
  for (int i = 0; i < a.rows; ++i)
    for (int p = a.ptr[i]; p < a.ptr[i + 1]; ++p) {
      const int q = next[a.idx[p]]++;
      t.idx[q] = i;
      t.val[q] = a.val[p];
    }
  return t;
}

void Tape::append(const Tape& t) {
  const int64_t ib = int64_t(idx.size()), vb = int64_t(val.size());
  types.insert(types.end(), t.types.begin(), t.types.end());
  idx.insert(idx.end(), t.idx.begin(), t.idx.end());
  val.insert(val.end(), t.val.begin(), t.val.end());
  for (size_t k = 1; k < t.is.size(); ++k) {
    is.push_back(ib + t.is[k]);
    vs.push_back(vb + t.vs[k]);
  }
}

double det_sum(const std::vector<double>& v) {
  // Chunks of 2048: thread t of 256 sums elements t, t+256, ..., then a
  // halving tree in shared memory; chunk totals are added in chunk order.
  const size_t n = v.size();
  double total = 0.0;
  for (size_t base = 0; base < n; base += 2048) {
    double s[256];
    for (int t = 0; t < 256; ++t) {
      double acc = 0.0;
      for (size_t k = base + size_t(t); k < std::min(n, base + 2048); k += 256) acc += v[k];
      s[t] = acc;
    }
    for (int h = 128; h > 0; h >>= 1)
      for (int t = 0; t < h; ++t) s[t] = s[t] + s[t + h];
    total += s[0];
  }
  return total;
}

namespace {

// Live positions of one row in stored order (live_matrix.cuh:13-81 visits
// the same sequence as a physically compacted row).
inline void live_positions(const Csr& A, int row, const uint8_t* keep_col, std::vector<int>& out) {
  out.clear();
  for (int p = A.ptr[row]; p < A.ptr[row + 1]; ++p)
    if (!keep_col || keep_col[A.idx[p]]) out.push_back(p);
}

// Warp tree of the reference's medium-row kernels: shfl_down 16,8,4,2,1 with
// value = own + peer (gpu_presolve_kernels.cu:226-232).
template <class T>
T warp_tree_down(T v[32]) {
  for (int off = 16; off > 0; off >>= 1)
    for (int k = 0; k < off; ++k) v[k] = v[k] + v[k + off];
  return v[0];
}

// cub::BlockReduce<T,256> default (BLOCK_REDUCE_WARP_REDUCTIONS): each warp
// reduces with shfl offsets 1,2,4,8,16 (own + peer), then warp aggregates are
// added in warp order.
template <class T>
T cub_block_sum(const T* v256) {
  T agg[8];
  for (int w = 0; w < 8; ++w) {
    T v[32];
    for (int k = 0; k < 32; ++k) v[k] = v256[w * 32 + k];
    for (int off = 1; off < 32; off <<= 1)
      for (int k = 0; k + off < 32; ++k) v[k] = v[k] + v[k + off];
    agg[w] = v[0];
  }
  T total = agg[0];
  for (int w = 1; w < 8; ++w) total = total + agg[w];
  return total;
}

}  // namespace

void row_activity_summary(const Csr& A, const std::vector<double>& l, const std::vector<double>& u,
                          double zero_tol, const uint8_t* keep_row, const uint8_t* keep_col,
                          const int* live_degrees, double* min_fin, double* max_fin,
                          int* min_inf, int* max_inf) {
  row_activity_impl(A, l, u, zero_tol, keep_row, keep_col, live_degrees, min_fin, max_fin, min_inf, max_inf, false);
}

void row_plain_minmax(const Csr& A, const std::vector<double>& l, const std::vector<double>& u,
                      const uint8_t* keep_row, const uint8_t* keep_col, const int* live_degrees,
                      double* row_min, double* row_max) {
  // The redundant-row sums (rule_infeasible_and_redundant_rows.cu:46-156):
  // plain sums of a*l / a*u over live entries, infinities propagate, same
  // bucket association as the activity summary.
  std::vector<int> ni(static_cast<size_t>(A.rows)), pi(static_cast<size_t>(A.rows));
  row_activity_impl(A, l, u, 0.0, keep_row, keep_col, live_degrees, row_min, row_max, ni.data(), pi.data(), true);
}

void row_activity_impl(const Csr& A, const std::vector<double>& l, const std::vector<double>& u,
                       double zero_tol, const uint8_t* keep_row, const uint8_t* keep_col,
                       const int* live_degrees, double* min_fin, double* max_fin,
                       int* min_inf, int* max_inf, bool plain) {
  // compute_row_activity_summary (gpu_presolve_kernels.cu:96-148,194-245,744-787):
  // rows of (live) length <= 8 sum sequentially; 9..1024 use 32 lane-strided
  // partials and a shfl_down tree; > 1024 use 256 partials and cub BlockReduce.
  std::vector<int> pos;
  for (int i = 0; i < A.rows; ++i) {
    const int len = live_degrees ? live_degrees[i] : A.ptr[i + 1] - A.ptr[i];
    const bool active = !keep_row || keep_row[i];
    if (active) live_positions(A, i, keep_col, pos); else pos.clear();
    auto term = [&](int p, double& lo, double& hi, int& ni, int& pi) {
      const double a = A.val[p];
      if (plain) {
        const int col = A.idx[p];
        lo += a >= 0.0 ? a * l[col] : a * u[col];
        hi += a >= 0.0 ? a * u[col] : a * l[col];
        return;
      }
      if (std::fabs(a) <= zero_tol) return;
      const int col = A.idx[p];
      const double tlo = a >= 0.0 ? a * l[col] : a * u[col];
      const double thi = a >= 0.0 ? a * u[col] : a * l[col];
      if (std::isfinite(tlo)) lo += tlo; else if (tlo < 0.0) ++ni;
      if (std::isfinite(thi)) hi += thi; else if (thi > 0.0) ++pi;
    };
    double lo = 0.0, hi = 0.0;
    int ni = 0, pi = 0;
    if (len <= 8) {
      for (int p : pos) term(p, lo, hi, ni, pi);
    } else {
      const int W = len <= 1024 ? 32 : 256;
      std::vector<double> plo(W, 0.0), phi(W, 0.0);
      std::vector<int> pni(W, 0), ppi(W, 0);
      for (size_t r = 0; r < pos.size(); ++r) {
        const int k = int(r % size_t(W));
        term(pos[r], plo[k], phi[k], pni[k], ppi[k]);
      }
      if (W == 32) {
        lo = warp_tree_down(plo.data());
        hi = warp_tree_down(phi.data());
        ni = warp_tree_down(pni.data());
        pi = warp_tree_down(ppi.data());
      } else {
        lo = cub_block_sum(plo.data());
        hi = cub_block_sum(phi.data());
        ni = cub_block_sum(pni.data());
        pi = cub_block_sum(ppi.data());
      }
    }
    min_fin[i] = lo;
    max_fin[i] = hi;
    min_inf[i] = ni;
    max_inf[i] = pi;
  }
}

void live_stats(const Csr& M, const uint8_t* keep_outer, const uint8_t* keep_inner, int* degree,
                uint8_t* empty, uint8_t* singleton, int* support, double* coefficient,
                int64_t* total) {
  // live_stats_kernel (gpu_presolve_kernels.cu:422-490): the singleton support
  // is the (unique) live entry; stored zeros count as entries.
  for (int r = 0; r < M.rows; ++r) {
    const bool active = !keep_outer || keep_outer[r];
    int count = 0, position = -1;
    if (active)
      for (int p = M.ptr[r]; p < M.ptr[r + 1]; ++p) {
        if (keep_inner && !keep_inner[M.idx[p]]) continue;
        ++count;
        position = p;
      }
    if (degree) degree[r] = count;
    if (empty) empty[r] = active && count == 0;
    if (singleton) singleton[r] = active && count == 1;
    if (support) support[r] = count == 1 ? M.idx[position] : -1;
    if (coefficient) coefficient[r] = count == 1 ? M.val[position] : 0.0;
    if (total) *total += count;
  }
}

void col_max_abs(const Csr& AT, const uint8_t* keep_row, double* out) {
  // compute_col_max_abs (gpu_presolve_kernels.cu:150-167,247-271,789-809).
  for (int j = 0; j < AT.rows; ++j) {
    double v = 0.0;
    for (int p = AT.ptr[j]; p < AT.ptr[j + 1]; ++p)
      if (!keep_row || keep_row[AT.idx[p]]) v = std::fmax(v, std::fabs(AT.val[p]));
    out[j] = v;
  }
}

}  // namespace oracle
