// Runs the REFERENCE GPU-Preprocessor library (built from its sources by
// oracle/ref.mk into oracle/_ref/) on one LP file and exports what it
// produced, so tests on a CUDA machine can compare the engine's structure and
// values with the reference's own implementation.  TEST INFRASTRUCTURE ONLY.
//
// usage: ref_driver <lp.bin> <out_dir> [key=value ...] [--repeat K]
//        [--postsolve x.bin y.bin z.bin]
// LP file format: see gpp_b200/lpgen.py save_lp.  Outputs (raw little-endian):
// meta.txt, A_ptr/A_idx/A_val, AT_ptr/AT_idx/AT_val, c/l/u/AL/AU, row_map,
// col_map, fixed_idx/fixed_val, tape_types/tape_is/tape_vs/tape_idx/tape_val,
// ckpt_kind/ckpt_payload/ckpt_position (primal-recovery checkpoints),
// abs<k>_* (absolute-value recoveries; pattern in meta.txt), vp<k>_*
// (variable-pair recoveries), and (with
// --postsolve) x_org/y_org/z_org.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpu_preprocessor/gpu_preprocessor.hpp"
#include "gpu_preprocessor/presolve/device_recovery.hpp"

namespace gp = gpu_preprocessor;

static void ck(cudaError_t e, const char* w) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(w) + ": " + cudaGetErrorString(e));
}
template <class T>
static T* up(const std::vector<T>& v) {
  T* p = nullptr;
  ck(cudaMalloc(&p, sizeof(T) * (v.size() ? v.size() : 1)), "cudaMalloc");
  if (!v.empty()) ck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "h2d");
  return p;
}
template <class T>
static std::vector<T> down(const T* p, size_t n) {
  std::vector<T> v(n);
  if (n && p) ck(cudaMemcpy(v.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost), "d2h");
  return v;
}
template <class T>
static void save(const std::string& dir, const char* name, const std::vector<T>& v) {
  std::ofstream f(dir + "/" + name, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
}
template <class T>
static std::vector<T> load(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  const auto bytes = size_t(f.tellg());
  std::vector<T> v(bytes / sizeof(T));
  f.seekg(0);
  f.read(reinterpret_cast<char*>(v.data()), std::streamsize(bytes));
  return v;
}

int main(int argc, char** argv) {
  try {
    if (argc < 3) {
      std::cerr << "usage: ref_driver <lp.bin> <out_dir> [key=value ...] [--repeat K] [--postsolve x y z]\n";
      return 2;
    }
    const std::string in = argv[1], out = argv[2];
    gp::Parameters p;
    int repeat = 1;
    std::string xs, ys, zs;
    for (int a = 3; a < argc; ++a) {
      std::string s = argv[a];
      if (s == "--repeat") { repeat = std::stoi(argv[++a]); continue; }
      if (s == "--postsolve") { xs = argv[++a]; ys = argv[++a]; zs = argv[++a]; continue; }
      const auto eq = s.find('=');
      const std::string k = s.substr(0, eq);
      const double dv = std::stod(s.substr(eq + 1));
      const int v = static_cast<int>(dv);
#define FLAG(name) else if (k == #name) p.name = v != 0
      if (false) {}
      FLAG(enable_folding); FLAG(enable_presolve);
      FLAG(enable_infeasible_and_fixed_variables); FLAG(enable_empty_rows); FLAG(enable_singleton_rows);
      FLAG(enable_infeasible_and_redundant_rows); FLAG(enable_bound_strengthening);
      FLAG(enable_parallel_rows); FLAG(enable_empty_columns); FLAG(enable_singleton_columns);
      FLAG(enable_doubleton_equations); FLAG(enable_dual_fix); FLAG(enable_parallel_columns);
      FLAG(enable_structure_specific_rules); FLAG(enable_startup);
      FLAG(enable_column_domination); FLAG(enable_two_row_variable_elimination);
      FLAG(enable_zero_cost_product_variables); FLAG(enable_piecewise_linear_reformulation_variable_pair);
      FLAG(enable_piecewise_linear_reformulation_absolute_value);
      else if (k == "column_domination_min_fixed_cols") p.column_domination_min_fixed_cols = v;
      else if (k == "column_domination_min_candidate_ratio") p.column_domination_min_candidate_ratio = dv;
      else if (k == "max_iters") p.max_iters = v;
      else if (k == "max_time") p.max_time = dv;
      else if (k == "folding_tolerance") p.folding_tolerance = dv;
      else if (k == "doubleton_equations_scan") p.doubleton_equations_scan = v != 0;
      else if (k == "doubleton_equations_max_fill_in_proxy") p.doubleton_equations_max_fill_in_proxy = v;
      else if (k == "doubleton_equations_min_selected_per_batch") p.doubleton_equations_min_selected_per_batch = v;
      else if (k == "doubleton_equations_min_selected_ratio") p.doubleton_equations_min_selected_ratio = dv;
#define NUM(name) else if (k == #name) p.name = static_cast<decltype(p.name)>(dv)
      NUM(piecewise_linear_reformulation_variable_pair_epigraph_probe_pairs);
      NUM(piecewise_linear_reformulation_variable_pair_epigraph_min_pairs);
      NUM(piecewise_linear_reformulation_variable_pair_epigraph_min_potential_gain);
      NUM(piecewise_linear_reformulation_variable_pair_epigraph_min_actual_gain);
      NUM(piecewise_linear_reformulation_variable_pair_epigraph_max_tail_cols);
      NUM(piecewise_linear_reformulation_variable_pair_epigraph_max_quotient_terms_per_row);
      NUM(piecewise_linear_reformulation_variable_pair_shifted_antipodal_probe_pairs);
      NUM(piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs);
      NUM(piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_potential_gain);
      NUM(piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_actual_gain);
      NUM(piecewise_linear_reformulation_variable_pair_shifted_antipodal_max_quotient_terms_per_row);
      NUM(feasibility_tol);
#undef NUM
      else if (k == "piecewise_linear_reformulation_absolute_value_residual_bound_mode")
        p.piecewise_linear_reformulation_absolute_value_residual_bound_mode =
            static_cast<gp::presolve::PiecewiseLinearReformulationAbsoluteValueResidualBoundMode>(v);
      else if (k == "piecewise_linear_reformulation_absolute_value_residual_bound_as_free_min")
        p.piecewise_linear_reformulation_absolute_value_residual_bound_as_free_min = dv;
      else throw std::invalid_argument("unknown parameter " + k);
#undef FLAG
    }
    // Read the LP and build A^T on the host (rows of A^T in ascending order).
    std::ifstream f(in, std::ios::binary);
    char magic[8];
    f.read(magic, 8);
    if (std::memcmp(magic, "GPPLP001", 8)) throw std::runtime_error("bad LP file");
    int64_t m, n, nnz;
    double obj;
    f.read(reinterpret_cast<char*>(&m), 8);
    f.read(reinterpret_cast<char*>(&n), 8);
    f.read(reinterpret_cast<char*>(&nnz), 8);
    f.read(reinterpret_cast<char*>(&obj), 8);
    auto rd = [&](auto& v, size_t k) { v.resize(k); f.read(reinterpret_cast<char*>(v.data()), std::streamsize(k * sizeof(v[0]))); };
    std::vector<int> ptr, idx;
    std::vector<double> val, c, l, u, AL, AU;
    rd(ptr, size_t(m) + 1); rd(idx, size_t(nnz)); rd(val, size_t(nnz));
    rd(c, size_t(n)); rd(l, size_t(n)); rd(u, size_t(n)); rd(AL, size_t(m)); rd(AU, size_t(m));
    std::vector<int> tptr(static_cast<size_t>(n) + 1, 0), tidx(static_cast<size_t>(nnz));
    std::vector<double> tval(static_cast<size_t>(nnz));
    for (int64_t q = 0; q < nnz; ++q) tptr[size_t(idx[size_t(q)]) + 1]++;
    for (int64_t j = 0; j < n; ++j) tptr[size_t(j) + 1] += tptr[size_t(j)];
    std::vector<int> next(tptr.begin(), tptr.end() - 1);
    for (int64_t i = 0; i < m; ++i)
      for (int q = ptr[size_t(i)]; q < ptr[size_t(i) + 1]; ++q) {
        const int t = next[size_t(idx[size_t(q)])]++;
        tidx[size_t(t)] = int(i);
        tval[size_t(t)] = val[size_t(q)];
      }
    gp::DeviceLp lp;
    lp.A = {int(m), int(n), int(nnz), up(ptr), up(idx), up(val)};
    lp.AT = {int(n), int(m), int(nnz), up(tptr), up(tidx), up(tval)};
    lp.c = up(c); lp.l = up(l); lp.u = up(u); lp.AL = up(AL); lp.AU = up(AU);
    lp.obj_constant = obj;
    ck(cudaDeviceSynchronize(), "upload");

    std::vector<double> wall;
    gp::Summary s;
    for (int r = 0; r < repeat; ++r) {
      if (r) gp::free_summary(s);
      ck(cudaDeviceSynchronize(), "pre");
      const auto t0 = std::chrono::steady_clock::now();
      s = gp::preprocess(lp, p);
      ck(cudaDeviceSynchronize(), "post");
      wall.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }
    const auto& ps = s.presolve;
    std::ofstream meta(out + "/meta.txt");
    meta << std::setprecision(17);
    meta << "status " << (ps.has_infeasible ? "infeasible" : ps.has_unbounded ? "unbounded" : "ok") << "\n";
    meta << "folding_applied " << s.folding_applied << "\nfolded_rows " << s.folded_rows << "\nfolded_cols "
         << s.folded_cols << "\n";
    meta << "reduced_rows " << ps.reduced_rows << "\nreduced_cols " << ps.reduced_cols << "\nreduced_nnz "
         << ps.reduced_nnz << "\niterations " << ps.iterations << "\nhas_change " << ps.has_change
         << "\nobj_constant_delta " << ps.obj_constant_delta << "\nstopped_at_iteration_limit "
         << ps.stopped_at_iteration_limit << "\n";
    meta << "preprocessing_seconds " << s.preprocessing_seconds << "\npresolve_seconds " << ps.elapsed_seconds
         << "\nfolding_seconds " << s.folding.profile.total_seconds << "\n";
    meta << "wall_seconds";
    for (double w : wall) meta << " " << w;
    meta << "\n";
    const auto& L = ps.reduced_lp;
    if (!ps.has_infeasible && !ps.has_unbounded) {
      save(out, "A_ptr", down(L.A.rowPtr, size_t(L.A.rows) + 1));
      save(out, "A_idx", down(L.A.colVal, size_t(L.A.nnz)));
      save(out, "A_val", down(L.A.nzVal, size_t(L.A.nnz)));
      save(out, "AT_ptr", down(L.AT.rowPtr, size_t(L.AT.rows) + 1));
      save(out, "AT_idx", down(L.AT.colVal, size_t(L.AT.nnz)));
      save(out, "AT_val", down(L.AT.nzVal, size_t(L.AT.nnz)));
      save(out, "c", down(L.c, size_t(L.A.cols)));
      save(out, "l", down(L.l, size_t(L.A.cols)));
      save(out, "u", down(L.u, size_t(L.A.cols)));
      save(out, "AL", down(L.AL, size_t(L.A.rows)));
      save(out, "AU", down(L.AU, size_t(L.A.rows)));
    }
    if (s.folding_applied) {
      const auto map = gp::folding::copy_map_to_host(s.folding.map);
      save(out, "row_color", map.row_color_id);
      save(out, "col_color", map.col_color_id);
      save(out, "row_scale", map.row_scale);
      save(out, "col_scale", map.col_scale);
    }
    // Fills the record's host views; postsolve keeps using the device state.
    auto& record = const_cast<gp::presolve::PresolveRecordGpu&>(ps.record);
    gp::presolve::export_recovery_record(record);
    save(out, "row_map", record.row_red2org);
    save(out, "col_map", record.col_red2org);
    save(out, "fixed_idx", record.fixed_idx);
    save(out, "fixed_val", record.fixed_val);
    save(out, "tape_types", record.tape.types);
    save(out, "tape_is", record.tape.index_starts);
    save(out, "tape_vs", record.tape.value_starts);
    save(out, "tape_idx", record.tape.indices);
    save(out, "tape_val", record.tape.vals);
    // Primal-recovery checkpoints and the absolute-value recoveries.
    {
      std::vector<int> kinds, payloads;
      std::vector<long long> positions;
      for (const auto& c : record.primal_recovery_timeline) {
        kinds.push_back(int(c.kind));
        payloads.push_back(int(c.payload_index));
        positions.push_back((long long)c.tape_position);
      }
      save(out, "ckpt_kind", kinds);
      save(out, "ckpt_payload", payloads);
      save(out, "ckpt_position", positions);
      meta << "absolute_value_steps " << record.piecewise_linear_reformulation_absolute_value_recoveries.size()
           << "\n";
      meta << "variable_pair_steps " << record.piecewise_linear_reformulation_variable_pair_recoveries.size()
           << "\n";
      int v = 0;
      for (const auto& a : record.piecewise_linear_reformulation_variable_pair_recoveries) {
        const std::string p = "vp" + std::to_string(v++) + "_";
        save(out, (p + "plus").c_str(), a.plus_cols); save(out, (p + "minus").c_str(), a.minus_cols);
        save(out, (p + "root_plus").c_str(), a.root_plus_cols);
        save(out, (p + "root_minus").c_str(), a.root_minus_cols);
        save(out, (p + "plus_shift").c_str(), a.plus_shift);
        save(out, (p + "minus_shift").c_str(), a.minus_shift);
      }
      int k = 0;
      for (const auto& a : record.piecewise_linear_reformulation_absolute_value_recoveries) {
        const std::string p = "abs" + std::to_string(k++) + "_";
        meta << p << "pattern " << a.pattern << "\n";
        std::vector<int> st, se, pb, pf, ls, lt, ms, mstart{0}, mt;
        std::vector<double> sr, lf, mf;
        for (const auto& x : a.splits) { st.push_back(x.t_col); se.push_back(x.e_col); sr.push_back(x.rho); }
        for (const auto& x : a.outer_pairs) { pb.push_back(x.bound_col); pf.push_back(x.free_col); }
        for (const auto& x : a.linked_slacks) { ls.push_back(x.slack_col); lt.push_back(x.t_col); lf.push_back(x.factor); }
        for (const auto& g : a.max_slacks) {
          ms.push_back(g.slack_col);
          mt.insert(mt.end(), g.t_cols.begin(), g.t_cols.end());
          mf.insert(mf.end(), g.factors.begin(), g.factors.end());
          mstart.push_back(int(mt.size()));
        }
        save(out, (p + "split_t").c_str(), st); save(out, (p + "split_e").c_str(), se);
        save(out, (p + "split_rho").c_str(), sr);
        save(out, (p + "pair_bound").c_str(), pb); save(out, (p + "pair_free").c_str(), pf);
        save(out, (p + "link_slack").c_str(), ls); save(out, (p + "link_t").c_str(), lt);
        save(out, (p + "link_factor").c_str(), lf);
        save(out, (p + "max_slack").c_str(), ms); save(out, (p + "max_start").c_str(), mstart);
        save(out, (p + "max_t").c_str(), mt); save(out, (p + "max_factor").c_str(), mf);
      }
    }
    if (!xs.empty()) {
      auto x = load<double>(xs), y = load<double>(ys), z = load<double>(zs);
      double *dx = up(x), *dy = up(y), *dz = up(z);
      const auto t0 = std::chrono::steady_clock::now();
      auto sol = gp::postprocess(dx, dy, dz, s, lp);
      ck(cudaDeviceSynchronize(), "postprocess");
      meta << "postsolve_seconds " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
           << "\n";
      save(out, "x_org", sol.x);
      save(out, "y_org", sol.y);
      save(out, "z_org", sol.z);
    }
    gp::free_summary(s);
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_driver: " << e.what() << "\n";
    return 1;
  }
}
