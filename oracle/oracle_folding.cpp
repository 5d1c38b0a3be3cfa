// Oracle folding: colour refinement and the quotient LP, restated on the CPU.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
//
// Reference: run_folding (cpp/src/folding/folding.cu:69-133), refine_color
// (folding_refinement.cu:222-359), update_color_id (folding_kernels.cu:
// 165-210), reduce_size (folding_reduce.cu:244-565), build_device_map
// (folding_map.cu:106-249).  Signatures use std::log / std::cos, so they can
// differ from the device's in the last bits; the partitions they induce are
// the same except in the rare case of a value on a single-precision rounding
// boundary.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "oracle.hpp"

namespace oracle {

namespace {

uint64_t finalize(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
double unit_of(uint64_t x) {
  const double u = double(finalize(x) >> 11) * 0x1.0p-53;
  return u > 0.0 ? u : 0x1.0p-53;
}
uint64_t round_seed(int round, uint64_t side) { return finalize(uint64_t(round) ^ (side * 0x9e3779b97f4a7c15ULL)); }
double signature(uint64_t seed, int color) {
  const uint64_t c = uint64_t(color);
  const double u1 = unit_of(seed ^ (c * 0xbf58476d1ce4e5b9ULL));
  const double u2 = unit_of((seed + 0x9e3779b97f4a7c15ULL) ^ (c * 0x94d049bb133111ebULL));
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925286766559 * u2);
}

struct Side {
  int n = 0, colors = 1;
  std::vector<int> ids;
  std::vector<double> sig;
  // update_color_id (folding_kernels.cu:165-210).
  void update(const std::vector<double>& value, double tol, bool write_sig, uint64_t seed) {
    std::vector<int> perm(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) perm[size_t(i)] = i;
    std::vector<float> f(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) f[size_t(i)] = float(value[size_t(i)]);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
      if (ids[size_t(a)] != ids[size_t(b)]) return ids[size_t(a)] < ids[size_t(b)];
      return f[size_t(a)] < f[size_t(b)];
    });
    int id = 0;
    std::vector<int> next(static_cast<size_t>(n));
    for (int q = 0; q < n; ++q) {
      const int i = perm[size_t(q)];
      bool start = q == 0;
      if (!start) {
        const int j = perm[size_t(q - 1)];
        start = ids[size_t(i)] != ids[size_t(j)] || double(f[size_t(i)]) > double(f[size_t(j)]) + tol;
      }
      if (start) ++id;
      next[size_t(i)] = id;
    }
    ids.swap(next);
    colors = id;
    if (write_sig)
      for (int i = 0; i < n; ++i) sig[size_t(i)] = signature(seed, ids[size_t(i)]);
  }
};

std::vector<double> spmv(const Csr& M, const std::vector<double>& x) {
  std::vector<double> y(static_cast<size_t>(M.rows), 0.0);
  for (int r = 0; r < M.rows; ++r) {
    double acc = 0.0;
    for (int p = M.ptr[r]; p < M.ptr[r + 1]; ++p) acc += M.val[p] * x[size_t(M.idx[p])];
    y[size_t(r)] = acc;
  }
  return y;
}

bool too_little(const Side& r, const Side& c) {
  return double(r.colors) > 0.8 * double(r.n) && double(c.colors) > 0.8 * double(c.n);
}

bool exact_repeat_sum(double value, int count, double& sum) {
  if (value == 0.0) { sum = 0.0; return true; }
  if (std::isinf(value)) { sum = value; return true; }
  if (!std::isfinite(value) || count <= 0) return false;
  uint64_t bits;
  std::memcpy(&bits, &value, 8);
  bits &= 0x7fffffffffffffffULL;
  uint64_t mant = bits & 0xfffffffffffffULL;
  if (bits >> 52) mant |= 1ULL << 52;
  while (!(mant & 1ULL)) mant >>= 1;
  if (mant > (1ULL << 53) / uint32_t(count)) return false;
  const double product = value * double(count);
  if (!std::isfinite(product)) return false;
  sum = product;
  return true;
}

}  // namespace

Fold fold(const Lp& lp, double tol) {
  if (!std::isfinite(tol) || tol < 0.0) throw std::invalid_argument("folding tolerance must be finite and nonnegative");
  Fold F;
  F.rows = lp.m();
  F.cols = lp.n();
  if (lp.m() == 0 || lp.n() == 0) return F;
  Side R, C;
  R.n = lp.m(); R.ids.assign(size_t(R.n), 0); R.sig.assign(size_t(R.n), 0.0);
  C.n = lp.n(); C.ids.assign(size_t(C.n), 0); C.sig.assign(size_t(C.n), 0.0);
  R.update(lp.AL, tol, false, 0); R.update(lp.AU, tol, false, 0);
  C.update(lp.c, tol, false, 0); C.update(lp.l, tol, false, 0); C.update(lp.u, tol, false, 0);
  for (int i = 0; i < R.n; ++i) R.sig[size_t(i)] = signature(round_seed(0, 2), R.ids[size_t(i)]);
  for (int j = 0; j < C.n; ++j) C.sig[size_t(j)] = signature(round_seed(0, 5), C.ids[size_t(j)]);
  if (too_little(R, C)) return F;
  const int max_round = std::max(1, R.n + C.n);
  bool ok = true;
  for (int round = 1; round <= max_round; ++round) {
    const int pr = R.colors, pc = C.colors;
    C.update(spmv(lp.AT, R.sig), tol, true, round_seed(round, 1));
    R.update(spmv(lp.A, C.sig), tol, true, round_seed(round, 2));
    if (too_little(R, C)) { ok = false; break; }
    if (!(R.colors > pr || C.colors > pc)) break;
  }
  if (!ok || (R.colors == R.n && C.colors == C.n)) return F;
  const int mr = R.colors, nc = C.colors;
  std::vector<int> rcount(size_t(mr), 0), ccount(size_t(nc), 0);
  for (int i = 0; i < R.n; ++i) ++rcount[size_t(R.ids[size_t(i)] - 1)];
  for (int j = 0; j < C.n; ++j) ++ccount[size_t(C.ids[size_t(j)] - 1)];
  // Members of each colour in index order.
  auto members = [](const std::vector<int>& ids, int k) {
    std::vector<std::vector<int>> m(static_cast<size_t>(k));
    for (size_t i = 0; i < ids.size(); ++i) m[size_t(ids[i] - 1)].push_back(int(i));
    return m;
  };
  const auto rm = members(R.ids, mr), cm = members(C.ids, nc);
  // Folded A: entries keyed by colour pair, summed in entry order.
  std::vector<std::pair<uint64_t, int>> keyed;
  std::vector<double> weighted(static_cast<size_t>(lp.A.nnz()));
  for (int r = 0; r < lp.m(); ++r) {
    const int Rr = R.ids[size_t(r)];
    const double w = 1.0 / double(rcount[size_t(Rr - 1)]);
    for (int p = lp.A.ptr[r]; p < lp.A.ptr[r + 1]; ++p) {
      keyed.push_back({uint64_t(Rr - 1) * uint64_t(nc) + uint64_t(C.ids[size_t(lp.A.idx[p])] - 1), p});
      weighted[size_t(p)] = lp.A.val[p] * w;
    }
  }
  std::stable_sort(keyed.begin(), keyed.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  Csr A;
  A.rows = mr;
  A.cols = nc;
  A.ptr.assign(size_t(mr) + 1, 0);
  for (size_t q = 0; q < keyed.size();) {
    const uint64_t key = keyed[q].first;
    double sum = 0.0;
    for (; q < keyed.size() && keyed[q].first == key; ++q) sum += weighted[size_t(keyed[q].second)];
    if (std::fabs(sum) > tol) {
      A.idx.push_back(int(key % uint64_t(nc)));
      A.val.push_back(sum);
      ++A.ptr[size_t(key / uint64_t(nc)) + 1];
    }
  }
  for (int r = 0; r < mr; ++r) A.ptr[size_t(r) + 1] += A.ptr[size_t(r)];
  Lp out;
  out.A = A;
  out.AT = transpose(A);
  out.obj = lp.obj;
  auto sum_values = [&](const std::vector<int>& mem, const std::vector<double>& v) {
    bool constant = true;
    for (int i : mem) constant = constant && v[size_t(i)] == v[size_t(mem[0])];
    double s = 0.0;
    if (constant && exact_repeat_sum(v[size_t(mem[0])], int(mem.size()), s)) return s;
    s = 0.0;
    for (int i : mem) s += v[size_t(i)];
    return s;
  };
  auto average_bounds = [&](const std::vector<int>& mem, const std::vector<double>& lo, const std::vector<double>& hi,
                            double& lo_out, double& hi_out) {
    bool lc = true, hc = true;
    for (int i : mem) { lc = lc && lo[size_t(i)] == lo[size_t(mem[0])]; hc = hc && hi[size_t(i)] == hi[size_t(mem[0])]; }
    double ls = 0.0, hs = 0.0;
    const int k = int(mem.size());
    const bool le = lc && exact_repeat_sum(lo[size_t(mem[0])], k, ls);
    const bool he = hc && exact_repeat_sum(hi[size_t(mem[0])], k, hs);
    if (!(le && he)) {
      if (!le) ls = 0.0;
      if (!he) hs = 0.0;
      for (int i : mem) { if (!le) ls += lo[size_t(i)]; if (!he) hs += hi[size_t(i)]; }
    }
    lo_out = ls / double(k);
    hi_out = hs / double(k);
  };
  out.c.resize(size_t(nc)); out.l.resize(size_t(nc)); out.u.resize(size_t(nc));
  out.AL.resize(size_t(mr)); out.AU.resize(size_t(mr));
  for (int k = 0; k < nc; ++k) {
    out.c[size_t(k)] = sum_values(cm[size_t(k)], lp.c);
    average_bounds(cm[size_t(k)], lp.l, lp.u, out.l[size_t(k)], out.u[size_t(k)]);
  }
  for (int k = 0; k < mr; ++k) average_bounds(rm[size_t(k)], lp.AL, lp.AU, out.AL[size_t(k)], out.AU[size_t(k)]);
  F.applied = true;
  F.folded = std::move(out);
  F.row_color = R.ids;
  F.col_color = C.ids;
  F.row_scale.resize(size_t(R.n));
  F.col_scale.resize(size_t(C.n));
  for (int i = 0; i < R.n; ++i) F.row_scale[size_t(i)] = 1.0 / double(rcount[size_t(R.ids[size_t(i)] - 1)]);
  for (int j = 0; j < C.n; ++j) F.col_scale[size_t(j)] = 1.0 / double(ccount[size_t(C.ids[size_t(j)] - 1)]);
  return F;
}

}  // namespace oracle
