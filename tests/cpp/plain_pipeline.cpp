// A user program of the C++ layer (include/gpu_preprocessor/): it includes
// gpu_preprocessor/gpu_preprocessor.hpp exactly as a GPU-Preprocessor user
// does and calls preprocess / postprocess / free_summary plus the presolve
// and folding namespaces.  tests/test_cpp_layer.py compiles it and compares
// what it writes with the Python (ctypes) path on the same LP.
//
// usage: plain_pipeline defaults
//        plain_pipeline run <lp.bin> <out_dir> [field=value ...]
//        plain_pipeline fold <lp.bin> <out_dir>
// `defaults` checks PresolveParams{} against gpp_default_params (no GPU).
// `run` writes meta.txt, the recovery maps and tape, the folding map (when
// folding applied), the reduced solution it fed to postprocess (xr, yr, zr)
// and the recovered solution (x, y, z; and px, py, pz from the presolve-only
// path).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "gpu_preprocessor/gpu_preprocessor.hpp"

namespace gpp = gpu_preprocessor;
namespace ps = gpu_preprocessor::presolve;

static void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
static T* upload(const std::vector<T>& v) {
  T* p = nullptr;
  ck(cudaMalloc(&p, sizeof(T) * (v.empty() ? 1 : v.size())), "cudaMalloc");
  if (!v.empty()) ck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
  return p;
}

template <class T>
static std::vector<T> download(const T* p, std::size_t n) {
  std::vector<T> v(n);
  if (n) ck(cudaMemcpy(v.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost), "download");
  return v;
}

template <class T>
static void save(const std::string& dir, const char* name, const std::vector<T>& v) {
  std::ofstream f(dir + "/" + name, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
}

static int check_defaults() {
  const gpp_params mine = ps::detail::to_c(ps::PresolveParams{});
  gpp_params lib;
  gpp_default_params(&lib);
  int bad = 0;
#define GPP_CHECK_FIELD(type, name, value)                                         \
  if (std::memcmp(&mine.name, &lib.name, sizeof(mine.name)) != 0) {                \
    std::cerr << "default differs: " #name "\n";                                   \
    ++bad;                                                                         \
  }
  GPP_PRESOLVE_PARAM_FIELDS(GPP_CHECK_FIELD)
#undef GPP_CHECK_FIELD
  std::cout << (bad ? "defaults differ\n" : "defaults match\n");
  return bad ? 1 : 0;
}

static void set_param(ps::PresolveParams& p, const std::string& key, const std::string& text) {
  const double v = std::stod(text);
#define GPP_SET_FIELD(type, name, value)   \
  if (key == #name) {                      \
    p.name = static_cast<decltype(p.name)>(v); \
    return;                                \
  }
  GPP_PRESOLVE_PARAM_FIELDS(GPP_SET_FIELD)
#undef GPP_SET_FIELD
  throw std::invalid_argument("unknown parameter " + key);
}

struct HostLp {
  std::int64_t m = 0, n = 0, nnz = 0;
  double obj = 0.0;
  std::vector<NnzOffset> ptr, tptr;
  std::vector<std::int32_t> idx, tidx;
  std::vector<double> val, tval, c, l, u, AL, AU;
};

static HostLp read_lp(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  char magic[8];
  f.read(magic, 8);
  if (!f || std::memcmp(magic, "GPPLP001", 8) != 0) throw std::runtime_error("bad LP file " + path);
  HostLp lp;
  f.read(reinterpret_cast<char*>(&lp.m), 8);
  f.read(reinterpret_cast<char*>(&lp.n), 8);
  f.read(reinterpret_cast<char*>(&lp.nnz), 8);
  f.read(reinterpret_cast<char*>(&lp.obj), 8);
  auto rd = [&](auto& v, std::int64_t k) {
    v.resize(static_cast<std::size_t>(k));
    f.read(reinterpret_cast<char*>(v.data()), std::streamsize(k * std::int64_t(sizeof(v[0]))));
  };
  rd(lp.ptr, lp.m + 1); rd(lp.idx, lp.nnz); rd(lp.val, lp.nnz);
  rd(lp.c, lp.n); rd(lp.l, lp.n); rd(lp.u, lp.n); rd(lp.AL, lp.m); rd(lp.AU, lp.m);
  // A^T with rows of A in ascending order inside every column.
  lp.tptr.assign(static_cast<std::size_t>(lp.n) + 1, 0);
  for (auto j : lp.idx) ++lp.tptr[static_cast<std::size_t>(j) + 1];
  for (std::size_t j = 0; j < static_cast<std::size_t>(lp.n); ++j) lp.tptr[j + 1] += lp.tptr[j];
  std::vector<NnzOffset> next(lp.tptr.begin(), lp.tptr.end() - 1);
  lp.tidx.resize(static_cast<std::size_t>(lp.nnz));
  lp.tval.resize(static_cast<std::size_t>(lp.nnz));
  for (std::int64_t i = 0; i < lp.m; ++i)
    for (NnzOffset q = lp.ptr[static_cast<std::size_t>(i)]; q < lp.ptr[static_cast<std::size_t>(i) + 1]; ++q) {
      const auto at = static_cast<std::size_t>(next[static_cast<std::size_t>(lp.idx[static_cast<std::size_t>(q)])]++);
      lp.tidx[at] = static_cast<std::int32_t>(i);
      lp.tval[at] = lp.val[static_cast<std::size_t>(q)];
    }
  return lp;
}

static int run(const std::string& in, const std::string& out, const ps::PresolveParams& params) {
  const HostLp h = read_lp(in);
  gpp::DeviceLp lp;
  lp.A = {int(h.m), int(h.n), checked_nnz_offset(h.nnz), upload(h.ptr), upload(h.idx), upload(h.val)};
  lp.AT = {int(h.n), int(h.m), checked_nnz_offset(h.nnz), upload(h.tptr), upload(h.tidx), upload(h.tval)};
  lp.c = upload(h.c); lp.l = upload(h.l); lp.u = upload(h.u); lp.AL = upload(h.AL); lp.AU = upload(h.AU);
  lp.obj_constant = h.obj;

  gpp::Summary first = gpp::preprocess(lp, params);
  // Summaries move but do not copy; the moved-from one no longer owns anything.
  gpp::Summary summary = std::move(first);
  if (first.presolve.record.handle.record != nullptr) throw std::runtime_error("moved-from summary still owns");
  gpp::free_summary(first);

  const auto& p = summary.presolve;
  std::ofstream meta(out + "/meta.txt");
  meta << std::setprecision(17);
  meta << "original_rows " << summary.original_rows << "\noriginal_cols " << summary.original_cols
       << "\nfolded_rows " << summary.folded_rows << "\nfolded_cols " << summary.folded_cols
       << "\nfolding_applied " << summary.folding_applied << "\npresolve_enabled " << summary.presolve_enabled
       << "\npresolve_original_rows " << p.original_rows << "\npresolve_original_cols " << p.original_cols
       << "\nreduced_rows " << p.reduced_rows << "\nreduced_cols " << p.reduced_cols << "\nreduced_nnz "
       << p.reduced_nnz << "\niterations " << p.iterations << "\nhas_change " << p.has_change
       << "\nhas_infeasible " << p.has_infeasible << "\nhas_unbounded " << p.has_unbounded
       << "\nobj_constant_delta " << p.obj_constant_delta << "\nrecord_obj_new " << p.record.obj_constant_new
       << "\n";

  ps::PresolveRecordGpu& record = summary.presolve.record;
  ps::export_recovery_record(record);
  save(out, "row_map", record.row_red2org);
  save(out, "col_map", record.col_red2org);
  save(out, "fixed_idx", record.fixed_idx);
  save(out, "fixed_val", record.fixed_val);
  save(out, "tape_types", record.tape.types);
  save(out, "tape_is", record.tape.index_starts);
  save(out, "tape_vs", record.tape.value_starts);
  save(out, "tape_idx", record.tape.indices);
  save(out, "tape_val", record.tape.vals);
  // The piecewise-linear reformulations' checkpoints and payloads, and the
  // absolute-value steps applied to a fixed vector by the public restore.
  {
    std::vector<std::int32_t> kinds, payloads, st, se, vplus, vroot;
    std::vector<long long> positions;
    std::vector<double> sr, vshift;
    for (const auto& c : record.primal_recovery_timeline) {
      kinds.push_back(static_cast<std::int32_t>(c.kind));
      payloads.push_back(c.payload_index);
      positions.push_back(c.tape_position);
    }
    for (const auto& a : record.piecewise_linear_reformulation_absolute_value_recoveries)
      for (const auto& x : a.splits) {
        st.push_back(x.t_col);
        se.push_back(x.e_col);
        sr.push_back(x.rho);
      }
    for (const auto& a : record.piecewise_linear_reformulation_variable_pair_recoveries) {
      vplus.insert(vplus.end(), a.plus_cols.begin(), a.plus_cols.end());
      vroot.insert(vroot.end(), a.root_plus_cols.begin(), a.root_plus_cols.end());
      vshift.insert(vshift.end(), a.plus_shift.begin(), a.plus_shift.end());
    }
    save(out, "ckpt_kind", kinds);
    save(out, "ckpt_payload", payloads);
    save(out, "ckpt_position", positions);
    save(out, "abs_split_t", st);
    save(out, "abs_split_e", se);
    save(out, "abs_split_rho", sr);
    save(out, "vp_plus", vplus);
    save(out, "vp_root_plus", vroot);
    save(out, "vp_plus_shift", vshift);
    if (!record.piecewise_linear_reformulation_absolute_value_recoveries.empty()) {
      std::vector<double> xv(static_cast<std::size_t>(h.n));
      for (std::size_t j = 0; j < xv.size(); ++j) xv[j] = 0.5 * double(j % 9) - 1.0;
      double* dxv = upload(xv);
      ps::postsolve_restore_piecewise_linear_reformulation_absolute_value_gpu(
          dxv, record.piecewise_linear_reformulation_absolute_value_recoveries, lp.l);
      save(out, "restored", download(dxv, xv.size()));
      ck(cudaFree(dxv), "cudaFree");
    }
  }

  if (summary.folding_applied) {
    const auto map = gpp::folding::copy_map_to_host(summary.folding.map);
    save(out, "row_color", map.row_color_id);
    save(out, "col_color", map.col_color_id);
    save(out, "row_scale", map.row_scale);
    save(out, "col_scale", map.col_scale);
  }
  if (p.has_infeasible || p.has_unbounded) {
    gpp::free_summary(summary);
    return 0;
  }

  // A deterministic reduced point inside the reduced bounds, and arbitrary duals.
  const auto m1 = static_cast<std::size_t>(p.reduced_rows), n1 = static_cast<std::size_t>(p.reduced_cols);
  const auto l1 = download(p.reduced_lp.l, n1), u1 = download(p.reduced_lp.u, n1);
  std::vector<double> xr(n1), yr(m1), zr(n1);
  for (std::size_t j = 0; j < n1; ++j) {
    xr[j] = std::fmin(std::fmax(0.5 * double(j % 7), l1[j]), u1[j]);
    zr[j] = 0.25 * (double(j % 3) - 1.0);
  }
  for (std::size_t i = 0; i < m1; ++i) yr[i] = 0.125 * (double(i % 5) - 2.0);
  save(out, "xr", xr);
  save(out, "yr", yr);
  save(out, "zr", zr);
  double *dx = upload(xr), *dy = upload(yr), *dz = upload(zr);
  const gpp::Solution sol = gpp::postprocess(dx, dy, dz, summary, lp);
  save(out, "x", sol.x);
  save(out, "y", sol.y);
  save(out, "z", sol.z);
  const std::int32_t reduced_rows = p.reduced_rows, reduced_cols = p.reduced_cols;
  gpp::free_summary(summary);
  gpp::free_summary(summary);  // a second call is a no-op

  // The presolve-only path on the same input: its postsolve equals the
  // pipeline's whenever folding did not apply.
  ps::GpuPresolveSummary only = ps::run_gpu_presolve_with_reduced_lp(lp, params);
  if (!only.has_infeasible && !only.has_unbounded && only.reduced_rows == reduced_rows &&
      only.reduced_cols == reduced_cols) {
    ps::GpuPostsolveResult r = ps::postsolve_gpu(dx, dy, dz, only.record, &lp);
    save(out, "px", download(r.x_org, static_cast<std::size_t>(r.n0)));
    save(out, "py", download(r.y_org, static_cast<std::size_t>(r.m0)));
    save(out, "pz", download(r.z_org, static_cast<std::size_t>(r.n0)));
    ck(cudaFree(r.x_org), "cudaFree");
    ck(cudaFree(r.y_org), "cudaFree");
    ck(cudaFree(r.z_org), "cudaFree");
  }
  ps::free_gpu_presolve_reduced_lp(only);
  for (void* q : {static_cast<void*>(dx), static_cast<void*>(dy), static_cast<void*>(dz),
                  static_cast<void*>(lp.A.rowPtr), static_cast<void*>(lp.A.colVal), static_cast<void*>(lp.A.nzVal),
                  static_cast<void*>(lp.AT.rowPtr), static_cast<void*>(lp.AT.colVal),
                  static_cast<void*>(lp.AT.nzVal), static_cast<void*>(lp.c), static_cast<void*>(lp.l),
                  static_cast<void*>(lp.u), static_cast<void*>(lp.AL), static_cast<void*>(lp.AU)})
    ck(cudaFree(q), "cudaFree");
  return 0;
}

// folding::run_folding alone: sizes, the map (host copy and the device
// arrays of the summary), the folded model, and the unfold of a folded point.
static int fold(const std::string& in, const std::string& out) {
  const HostLp h = read_lp(in);
  gpp::DeviceLp lp;
  lp.A = {int(h.m), int(h.n), checked_nnz_offset(h.nnz), upload(h.ptr), upload(h.idx), upload(h.val)};
  lp.AT = {int(h.n), int(h.m), checked_nnz_offset(h.nnz), upload(h.tptr), upload(h.tidx), upload(h.tval)};
  lp.c = upload(h.c); lp.l = upload(h.l); lp.u = upload(h.u); lp.AL = upload(h.AL); lp.AU = upload(h.AU);
  lp.obj_constant = h.obj;
  gpp::folding::FoldingRunSummary f = gpp::folding::run_folding(lp, 1e-9);
  std::ofstream meta(out + "/meta.txt");
  meta << "applied " << f.applied << "\noriginal_rows " << f.original_rows << "\noriginal_cols " << f.original_cols
       << "\nfolded_rows " << f.folded_rows << "\nfolded_cols " << f.folded_cols << "\nowns_folded_lp "
       << f.owns_folded_lp << "\nfolded_nnz " << f.folded_lp.A.nnz << "\n";
  if (f.applied) {
    const auto map = gpp::folding::copy_map_to_host(f.map);
    save(out, "row_color", map.row_color_id);
    save(out, "col_color", map.col_color_id);
    save(out, "row_scale", map.row_scale);
    save(out, "col_scale", map.col_scale);
    const auto m0 = static_cast<std::size_t>(f.original_rows), n0 = static_cast<std::size_t>(f.original_cols);
    save(out, "dev_row_color", download(f.map.row_color_id, m0));
    save(out, "dev_col_scale", download(f.map.col_scale, n0));
    const auto mf = static_cast<std::size_t>(f.folded_rows), nf = static_cast<std::size_t>(f.folded_cols);
    save(out, "F_ptr", download(f.folded_lp.A.rowPtr, mf + 1));
    save(out, "F_idx", download(f.folded_lp.A.colVal, static_cast<std::size_t>(f.folded_lp.A.nnz)));
    save(out, "F_val", download(f.folded_lp.A.nzVal, static_cast<std::size_t>(f.folded_lp.A.nnz)));
    save(out, "F_c", download(f.folded_lp.c, nf));
    std::vector<double> xf(nf), yf(mf), zf(nf);
    for (std::size_t j = 0; j < nf; ++j) { xf[j] = double(j % 5); zf[j] = 0.5 * double(j % 3); }
    for (std::size_t i = 0; i < mf; ++i) yf[i] = double(i % 4) - 1.0;
    double *dx = upload(xf), *dy = upload(yf), *dz = upload(zf);
    const auto u = gpp::folding::unfold_solution_device_to_host(f.map, dx, dy, dz);
    save(out, "ux", u.x);
    save(out, "uy", u.y);
    save(out, "uz", u.z);
    for (double* q : {dx, dy, dz}) ck(cudaFree(q), "cudaFree");
  }
  gpp::folding::free_folded_lp(f);
  gpp::folding::free_folded_lp(f);  // a second call is a no-op
  if (f.owns_folded_lp || f.map.row_color_id != nullptr) throw std::runtime_error("free_folded_lp left state");
  for (void* q : {static_cast<void*>(lp.A.rowPtr), static_cast<void*>(lp.A.colVal), static_cast<void*>(lp.A.nzVal),
                  static_cast<void*>(lp.AT.rowPtr), static_cast<void*>(lp.AT.colVal),
                  static_cast<void*>(lp.AT.nzVal), static_cast<void*>(lp.c), static_cast<void*>(lp.l),
                  static_cast<void*>(lp.u), static_cast<void*>(lp.AL), static_cast<void*>(lp.AU)})
    ck(cudaFree(q), "cudaFree");
  return 0;
}

int main(int argc, char** argv) {
  try {
    if (argc >= 2 && std::string(argv[1]) == "defaults") return check_defaults();
    if (argc == 4 && std::string(argv[1]) == "fold") return fold(argv[2], argv[3]);
    if (argc < 4 || std::string(argv[1]) != "run") {
      std::cerr << "usage: plain_pipeline defaults | run <lp.bin> <out_dir> [field=value ...]\n";
      return 2;
    }
    ps::PresolveParams params;
    for (int a = 4; a < argc; ++a) {
      const std::string s = argv[a];
      const auto eq = s.find('=');
      if (eq == std::string::npos) throw std::invalid_argument("expected field=value: " + s);
      set_param(params, s.substr(0, eq), s.substr(eq + 1));
    }
    return run(argv[2], argv[3], params);
  } catch (const std::exception& e) {
    std::cerr << "plain_pipeline: " << e.what() << "\n";
    return 1;
  }
}
