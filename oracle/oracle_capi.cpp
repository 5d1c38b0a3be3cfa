// C entry points of the oracle for the Python test-suite (ctypes).
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <cstring>
#include <exception>
#include <string>

#include "oracle.hpp"

namespace {
thread_local std::string g_error;

oracle::Csr make_csr(int rows, int cols, const int* ptr, const int* idx, const double* val) {
  oracle::Csr a;
  a.rows = rows;
  a.cols = cols;
  a.ptr.assign(ptr, ptr + rows + 1);
  a.idx.assign(idx, idx + ptr[rows]);
  a.val.assign(val, val + ptr[rows]);
  return a;
}
}  // namespace

extern "C" {

struct orc_lp {
  int32_t m, n;
  const int32_t* ptr;
  const int32_t* idx;
  const double* val;
  const int32_t* at_ptr;
  const int32_t* at_idx;
  const double* at_val;
  const double *c, *AL, *AU, *l, *u;
  double obj;
};

struct orc_result {
  oracle::Result r;
  oracle::Lp original;
  oracle::Fold fold;
};

const char* orc_last_error() { return g_error.c_str(); }

static oracle::Lp to_lp(const orc_lp* h) {
  oracle::Lp lp;
  lp.A = make_csr(h->m, h->n, h->ptr, h->idx, h->val);
  lp.AT = make_csr(h->n, h->m, h->at_ptr, h->at_idx, h->at_val);
  lp.c.assign(h->c, h->c + h->n);
  lp.l.assign(h->l, h->l + h->n);
  lp.u.assign(h->u, h->u + h->n);
  lp.AL.assign(h->AL, h->AL + h->m);
  lp.AU.assign(h->AU, h->AU + h->m);
  lp.obj = h->obj;
  return lp;
}

int orc_presolve(const orc_lp* h, const gpp_params* p, orc_result** out) {
  // run_gpu_presolve_with_folding (folding.cu:172-213): fold first when
  // enabled, then presolve whichever model results.
  try {
    auto* res = new orc_result;
    res->original = to_lp(h);
    if (p->enable_folding) res->fold = oracle::fold(res->original, p->folding_tolerance);
    const oracle::Lp& input = res->fold.applied ? res->fold.folded : res->original;
    res->r = oracle::presolve(input, *p);
    auto& s = res->r.summary;
    s.folding_applied = res->fold.applied ? 1 : 0;
    s.original_rows = res->original.m();
    s.original_cols = res->original.n();
    s.folded_rows = input.m();
    s.folded_cols = input.n();
    *out = res;
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 4;
  }
}

void orc_free(orc_result* r) { delete r; }

void orc_summary(const orc_result* r, gpp_summary* s) { *s = r->r.summary; }

// Reduced LP sizes and arrays (host copies).
void orc_reduced(const orc_result* r, int32_t* ptr, int32_t* idx, double* val, int32_t* at_ptr,
                 int32_t* at_idx, double* at_val, double* c, double* AL, double* AU, double* l,
                 double* u, double* obj) {
  const auto& L = r->r.reduced;
  auto cp = [](auto* dst, const auto& v) { if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0])); };
  cp(ptr, L.A.ptr); cp(idx, L.A.idx); cp(val, L.A.val);
  cp(at_ptr, L.AT.ptr); cp(at_idx, L.AT.idx); cp(at_val, L.AT.val);
  cp(c, L.c); cp(AL, L.AL); cp(AU, L.AU); cp(l, L.l); cp(u, L.u);
  if (obj) *obj = L.obj;
}

void orc_maps(const orc_result* r, int32_t* rows, int32_t* cols) {
  const auto& R = r->r.record;
  if (rows && !R.rows.empty()) std::memcpy(rows, R.rows.data(), R.rows.size() * 4);
  if (cols && !R.cols.empty()) std::memcpy(cols, R.cols.data(), R.cols.size() * 4);
}

void orc_tape_sizes(const orc_result* r, int64_t* records, int64_t* indices, int64_t* values,
                    int64_t* fixed) {
  const auto& R = r->r.record;
  *records = R.tape.count();
  *indices = int64_t(R.tape.idx.size());
  *values = int64_t(R.tape.val.size());
  *fixed = int64_t(R.fixed_idx.size());
}

void orc_tape(const orc_result* r, int32_t* types, int64_t* is, int64_t* vs, int32_t* idx,
              double* val, int32_t* fixed_idx, double* fixed_val) {
  const auto& R = r->r.record;
  auto cp = [](auto* dst, const auto& v) { if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0])); };
  cp(types, R.tape.types); cp(is, R.tape.is); cp(vs, R.tape.vs); cp(idx, R.tape.idx); cp(val, R.tape.val);
  cp(fixed_idx, R.fixed_idx); cp(fixed_val, R.fixed_val);
}

// copy_map_to_host (folding_map.cu:250-270); returns 1 when folding applied.
int orc_fold_map(const orc_result* r, int32_t* row_color, int32_t* col_color, double* row_scale, double* col_scale) {
  const auto& f = r->fold;
  if (!f.applied) return 0;
  auto cp = [](auto* dst, const auto& v) { if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0])); };
  cp(row_color, f.row_color); cp(col_color, f.col_color); cp(row_scale, f.row_scale); cp(col_scale, f.col_scale);
  return 1;
}

int orc_trace_count(const orc_result* r) { return int(r->r.trace.size()); }
const char* orc_trace(const orc_result* r, int k) { return r->r.trace[size_t(k)].c_str(); }

int orc_postsolve(const orc_result* r, const double* x_red, const double* y_red, const double* z_red,
                  double* x, double* y, double* z) {
  try {
    if (!r->fold.applied) {
      oracle::postsolve(r->r, r->original, x_red, y_red, z_red, x, y, z);
      return 0;
    }
    // postsolve_and_unfold_to_host (folding.cu:215-261): postsolve on the
    // folded model, then x_j = x_f[C(j)], y_i = y_f[R(i)]/|R|, z_j = z_f[C(j)]/|C|.
    const oracle::Lp& F = r->fold.folded;
    std::vector<double> xf(static_cast<size_t>(F.n())), yf(static_cast<size_t>(F.m())), zf(static_cast<size_t>(F.n()));
    oracle::postsolve(r->r, F, x_red, y_red, z_red, xf.data(), yf.data(), zf.data());
    const auto& fd = r->fold;
    for (int j = 0; j < fd.cols; ++j) {
      const int k = fd.col_color[size_t(j)] - 1;
      if (x) x[j] = xf[size_t(k)];
      if (z) z[j] = zf[size_t(k)] * fd.col_scale[size_t(j)];
    }
    if (y)
      for (int i = 0; i < fd.rows; ++i) y[i] = yf[size_t(fd.row_color[size_t(i)] - 1)] * fd.row_scale[size_t(i)];
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 4;
  }
}

// Kernel-level oracles.
void orc_row_activity_summary(int m, int n, const int32_t* ptr, const int32_t* idx, const double* val,
                              const double* l, const double* u, double zero_tol,
                              const uint8_t* keep_row, const uint8_t* keep_col,
                              const int32_t* live_degrees, double* min_fin, double* max_fin,
                              int32_t* min_inf, int32_t* max_inf) {
  auto A = make_csr(m, n, ptr, idx, val);
  std::vector<double> L(l, l + n), U(u, u + n);
  oracle::row_activity_summary(A, L, U, zero_tol, keep_row, keep_col, live_degrees, min_fin, max_fin,
                               min_inf, max_inf);
}

void orc_live_stats(int rows, int cols, const int32_t* ptr, const int32_t* idx, const double* val,
                    const uint8_t* keep_outer, const uint8_t* keep_inner, int32_t* degree,
                    uint8_t* empty, uint8_t* singleton, int32_t* support, double* coefficient,
                    int64_t* total) {
  auto M = make_csr(rows, cols, ptr, idx, val);
  oracle::live_stats(M, keep_outer, keep_inner, degree, empty, singleton, support, coefficient, total);
}

void orc_col_max_abs(int rows, int cols, const int32_t* ptr, const int32_t* idx, const double* val,
                     const uint8_t* keep_row, double* out) {
  auto M = make_csr(rows, cols, ptr, idx, val);
  oracle::col_max_abs(M, keep_row, out);
}

uint64_t orc_row_hash(int m, int n, const int32_t* ptr, const int32_t* idx, const double* val,
                      int row, const uint8_t* keep_col, int mode) {
  auto A = make_csr(m, n, ptr, idx, val);
  return oracle::row_hash(A, row, keep_col, mode);
}

double orc_det_sum(const double* v, int64_t n) { return oracle::det_sum(std::vector<double>(v, v + n)); }

}  // extern "C"
