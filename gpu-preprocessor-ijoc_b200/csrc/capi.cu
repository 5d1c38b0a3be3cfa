// extern "C" boundary (include/gpp.h).  Every entry point catches C++
// exceptions and maps them to the status codes the header documents; the C++
// API in include/gpu_preprocessor/ maps them back to the reference's
// exception types.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <cmath>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "folding.hpp"
#include "presolve.hpp"
#include "schedule_mlp.hpp"
#include "mps_reader.hpp"

#include <filesystem>
#include <fstream>
#include <iomanip>
#include "sort.hpp"

struct gpp_mps_model {
  gpp::MpsModel m;
};

struct gpp_schedule_model {
  std::unique_ptr<gpp::MlpSchedule> policy;
};

struct gpp_record {
  gpp::PresolveOutput out;
  gpp::FoldingResult folding;
  bool presolve_enabled = true;
};

namespace gpp {
const char* last_error();
}

using gpp::check;

namespace {

constexpr int kDefaultBatchWorkers = 8;
constexpr int kAutotuneSample = 32;

// A batch whose items failed: carries the first failing item's status (the
// message is already set).
struct BatchFailure {
  int status;
};

template <class F>
int guarded(F f) {
  try {
    int dev = 0;
    if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0) {
      cudaGetLastError();
      gpp::set_last_error("no CUDA device is available to the presolve engine");
      return GPP_ERR_NO_DEVICE;
    }
    f();
    gpp::set_last_error("");
    return GPP_OK;
  } catch (const gpp::CudaError& e) {
    gpp::set_last_error(e.what());
    return GPP_ERR_CUDA;
  } catch (const std::length_error& e) {
    gpp::set_last_error(e.what());
    return GPP_ERR_LENGTH;
  } catch (const std::invalid_argument& e) {
    gpp::set_last_error(e.what());
    return GPP_ERR_INVALID;
  } catch (const std::exception& e) {
    gpp::set_last_error(e.what());
    return GPP_ERR_RUNTIME;
  } catch (const BatchFailure& f) {
    return f.status;
  }
}

void validate_lp(const gpp_lp& lp) {
  if (lp.A.rows < 0 || lp.A.cols < 0 || lp.A.nnz < 0) throw std::invalid_argument("negative LP dimensions");
  if (lp.AT.rows != lp.A.cols || lp.AT.cols != lp.A.rows || lp.AT.nnz != lp.A.nnz)
    throw std::invalid_argument("AT must be the transpose of A (dimension/nnz mismatch)");
  if ((lp.A.cols && (!lp.c || !lp.l || !lp.u)) || (lp.A.rows && (!lp.AL || !lp.AU)) || !lp.A.rowPtr ||
      !lp.AT.rowPtr || (lp.A.nnz && (!lp.A.colVal || !lp.A.nzVal || !lp.AT.colVal || !lp.AT.nzVal)))
    throw std::invalid_argument("LP device pointer missing");
}

void fill_summary(gpp_summary* s, gpp_record* rec, double preprocessing_seconds) {
  const gpp::PresolveOutput& o = rec->out;
  *s = gpp_summary{};
  s->original_rows = o.original_rows;
  s->original_cols = o.original_cols;
  s->reduced_rows = o.reduced_rows;
  s->reduced_cols = o.reduced_cols;
  s->reduced_nnz = o.reduced_nnz;
  s->iterations = o.iterations;
  s->stopped_at_iteration_limit = o.stopped_at_iteration_limit;
  s->has_change = o.has_change;
  s->has_infeasible = o.has_infeasible;
  s->has_unbounded = o.has_unbounded;
  s->presolve_enabled = rec->presolve_enabled;
  s->folding_applied = rec->folding.applied;
  s->owns_reduced_lp = o.owns_reduced;
  s->elapsed_seconds = o.elapsed_seconds;
  s->preprocessing_seconds = preprocessing_seconds;
  s->obj_constant_delta = o.obj_constant_delta;
  // FoldingPipelineSummary (folding_structs.hpp:94-109): the original sizes
  // are the caller's model, the folded sizes what presolve ran on.
  if (rec->folding.applied) {
    s->original_rows = rec->folding.original_rows;
    s->original_cols = rec->folding.original_cols;
  }
  s->folded_rows = rec->folding.applied ? rec->folding.folded_rows : s->original_rows;
  s->folded_cols = rec->folding.applied ? rec->folding.folded_cols : s->original_cols;
  const gpp::WorkingLp& r = o.reduced;
  s->reduced_lp = gpp_lp{{r.A.rows, r.A.cols, r.A.nnz, r.A.ptr, r.A.idx, r.A.val},
                         {r.AT.rows, r.AT.cols, r.AT.nnz, r.AT.ptr, r.AT.idx, r.AT.val},
                         r.c, r.AL, r.AU, r.l, r.u, r.obj, 0, nullptr};
  s->record = rec;
}

void identity_output(const gpp_lp& lp, gpp::PresolveOutput& o) {
  // run_optional_gpu_presolve with enable_presolve = false (folding.cu:145-170).
  o.original_rows = o.reduced_rows = lp.A.rows;
  o.original_cols = o.reduced_cols = lp.A.cols;
  o.reduced_nnz = lp.A.nnz;
  gpp::init_record(o.record, lp.A.rows, lp.A.cols);
  o.reduced.A = gpp::DevCsr{lp.A.rows, lp.A.cols, lp.A.nnz, lp.A.rowPtr, lp.A.colVal, lp.A.nzVal};
  o.reduced.AT = gpp::DevCsr{lp.AT.rows, lp.AT.cols, lp.AT.nnz, lp.AT.rowPtr, lp.AT.colVal, lp.AT.nzVal};
  o.reduced.c = lp.c; o.reduced.AL = lp.AL; o.reduced.AU = lp.AU; o.reduced.l = lp.l; o.reduced.u = lp.u;
  o.reduced.obj = lp.obj_constant;
  o.owns_reduced = false;
}

// The body of gpp_preprocess.  `device_sync` waits for all work on the
// device before the timer starts, as the reference's pipeline timing does;
// the batched form skips it so that its workers do not wait on each other.
void preprocess_into(const gpp_lp* lp, const gpp_params* params, gpp_summary* out, bool device_sync,
                     gpp::SchedulePolicy* policy = nullptr, std::vector<gpp::RoundRecord>* trace = nullptr) {
  if (!lp || !params || !out) throw std::invalid_argument("null argument");
  validate_lp(*lp);
  auto rec = std::make_unique<gpp_record>();
  rec->presolve_enabled = params->enable_presolve != 0;
  gpp::ctx().sync("before preprocessing timer");
  if (device_sync) check(cudaDeviceSynchronize(), "before preprocessing timer");
  const auto t0 = std::chrono::steady_clock::now();
  if (params->enable_folding) gpp::run_folding(*lp, params->folding_tolerance, rec->folding);
  const gpp_lp& input = rec->folding.applied ? rec->folding.folded : *lp;
  if (params->enable_presolve) gpp::run_presolve(input, *params, rec->out, policy, trace);
  else identity_output(input, rec->out);
  gpp::ctx().sync("preprocessing completion");
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  fill_summary(out, rec.get(), secs);
  rec.release();
}

// The body of gpp_postprocess.
void postprocess_into(const double* x_red, const double* y_red, const double* z_red, const gpp_summary* summary,
                      const gpp_lp* original, double* x_out, double* y_out, double* z_out) {
  if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
  const gpp_record* rec = summary->record;
  auto s = gpp::ctx().stream;
  const int n0 = summary->original_cols, m0 = summary->original_rows;
  if (!rec->presolve_enabled && !rec->folding.applied) {
    auto copy = [&](double* dst, const double* src, int n) {
      if (dst && src && n) check(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "copy identity");
    };
    copy(x_out, x_red, n0); copy(y_out, y_red, m0); copy(z_out, z_red, n0);
    gpp::ctx().sync("identity postprocess");
    return;
  }
  const int pn = rec->out.record.n0, pm = rec->out.record.m0;
  gpp::DBuf<double> x(size_t(std::max(pn, 1)), s), y(size_t(std::max(pm, 1)), s), z(size_t(std::max(pn, 1)), s);
  if (!rec->presolve_enabled) {
    if (pn) { check(cudaMemcpyAsync(x.p, x_red, sizeof(double) * pn, cudaMemcpyDeviceToDevice, s), "x");
              check(cudaMemcpyAsync(z.p, z_red, sizeof(double) * pn, cudaMemcpyDeviceToDevice, s), "z"); }
    if (pm) check(cudaMemcpyAsync(y.p, y_red, sizeof(double) * pm, cudaMemcpyDeviceToDevice, s), "y");
  } else {
    const gpp_lp* model = rec->folding.applied ? &rec->folding.folded : original;
    gpp::run_postsolve(rec->out, x_red, y_red, z_red, model, x.p, y.p, z.p);
  }
  if (rec->folding.applied) {
    gpp::unfold_to_host(rec->folding, x.p, y.p, z.p, x_out, y_out, z_out);
  } else {
    if (x_out && pn) check(cudaMemcpyAsync(x_out, x.p, sizeof(double) * pn, cudaMemcpyDeviceToHost, s), "x d2h");
    if (y_out && pm) check(cudaMemcpyAsync(y_out, y.p, sizeof(double) * pm, cudaMemcpyDeviceToHost, s), "y d2h");
    if (z_out && pn) check(cudaMemcpyAsync(z_out, z.p, sizeof(double) * pn, cudaMemcpyDeviceToHost, s), "z d2h");
  }
  gpp::ctx().sync("postprocess");
}

// ---- batched form ----------------------------------------------------------
// A persistent pool of host threads.  Each thread keeps its own engine context
// (stream, schedules, status buffer), so LPs given to different threads run
// concurrently on the GPU and their host round-trips overlap.  Threads live
// until process exit: their contexts are created once, not per batch.
class WorkerPool {
 public:
  static WorkerPool& get() {
    static WorkerPool* pool = new WorkerPool;   // never destroyed: detached threads use it until exit
    return *pool;
  }

  // Runs task(order[0]), task(order[1]), ... on `workers` threads (the caller
  // is one of them), each item exactly once, every thread with `device`
  // current.  One batch at a time.
  void run(int workers, int device, const std::vector<int>& order, const std::function<void(int)>& task) {
    std::lock_guard<std::mutex> one_batch(batch_mutex_);
    workers = std::max(1, workers);
    {
      std::unique_lock<std::mutex> lock(m_);
      while (int(threads_) < workers - 1) {
        std::thread([this, id = int(threads_)] { loop(id); }).detach();
        ++threads_;
      }
      order_ = &order;
      task_ = &task;
      device_ = device;
      next_.store(0);
      active_ = workers - 1;
      running_ = workers - 1;
      ++generation_;
    }
    cv_.notify_all();
    drain();
    std::unique_lock<std::mutex> lock(m_);
    done_.wait(lock, [this] { return running_ == 0; });
    order_ = nullptr;
    task_ = nullptr;
  }

 private:
  void drain() {
    for (size_t i = next_.fetch_add(1); i < order_->size(); i = next_.fetch_add(1)) (*task_)((*order_)[i]);
  }
  void loop(int id) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lock(m_);
        cv_.wait(lock, [&] { return generation_ != seen; });
        seen = generation_;
        if (id >= active_) continue;
      }
      cudaSetDevice(device_);
      drain();
      std::lock_guard<std::mutex> lock(m_);
      if (--running_ == 0) done_.notify_all();
    }
  }

  std::mutex batch_mutex_, m_;
  std::condition_variable cv_, done_;
  size_t threads_ = 0;
  uint64_t generation_ = 0;
  int active_ = 0, running_ = 0, device_ = 0;
  std::atomic<size_t> next_{0};
  const std::vector<int>* order_ = nullptr;
  const std::function<void(int)>* task_ = nullptr;
};

// LP indices, largest nnz first (longest jobs start first, so the last
// finishers are short ones).
std::vector<int> largest_first(const gpp_lp* lps, int32_t count) {
  std::vector<int> order(static_cast<size_t>(count));
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return lps[a].A.nnz > lps[b].A.nnz; });
  return order;
}

// Runs one item per LP under the status mapping of the plain entry points;
// returns GPP_OK or the first failing status in LP order, whose message
// becomes the caller's last error.
int run_batch(int32_t count, int workers, const std::vector<int>& order, int32_t* status,
              const std::function<void(int)>& body) {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  std::vector<int32_t> st(static_cast<size_t>(count), GPP_OK);
  std::vector<std::string> msg(static_cast<size_t>(count));
  WorkerPool::get().run(workers, dev, order, [&](int k) {
    st[size_t(k)] = guarded([&] { body(k); });
    if (st[size_t(k)] != GPP_OK) msg[size_t(k)] = gpp::last_error();
  });
  if (status) std::copy(st.begin(), st.end(), status);
  for (int32_t k = 0; k < count; ++k)
    if (st[size_t(k)] != GPP_OK) {
      gpp::set_last_error("LP " + std::to_string(k) + ": " + msg[size_t(k)]);
      return st[size_t(k)];
    }
  return GPP_OK;
}

}  // namespace

extern "C" {

void gpp_default_params(gpp_params* p) {
  *p = gpp_params{};
  p->max_iters = 512;
  p->max_time = HUGE_VAL;
  p->verbose = 0;
  p->record_postsolve_tape = 1;
  p->record_postsolve_tape_cpu = 0;
  p->enable_presolve = 1;
  p->enable_folding = 1;
  p->folding_tolerance = 1.0e-8;
  p->feasibility_tol = 1.0e-6;
  p->bound_tol = 1.0e-6;
  p->zero_tol = 1.0e-10;
  p->bound_strengthening_upper_relaxation_factor = 1.0;
  p->bound_strengthening_max_rounds = 64;
  p->bound_strengthening_max_bound_only_rounds = 64;
  p->bound_strengthening_preserve_free_zero_cost = 1;
  p->doubleton_equations_max_fill_in_proxy = 96;
  p->doubleton_equations_scan = 1;
  p->doubleton_equations_min_selected_per_batch = 256;
  p->doubleton_equations_min_selected_ratio = 0.005;
  p->doubleton_equations_max_batch_rounds = 0;
  p->doubleton_equations_max_time = 0.0;
  p->enable_infeasible_and_fixed_variables = 1;
  p->enable_empty_rows = 1;
  p->enable_singleton_rows = 1;
  p->enable_infeasible_and_redundant_rows = 1;
  p->enable_bound_strengthening = 1;
  p->enable_parallel_rows = 1;
  p->enable_empty_columns = 1;
  p->enable_singleton_columns = 1;
  p->enable_doubleton_equations = 1;
  p->enable_dual_fix = 1;
  p->dual_fix_max_nonzero_cost_col_degree = 128;
  p->enable_parallel_columns = 1;
  p->parallel_columns_max_abs_ratio = 2.0;
  p->parallel_columns_scale_guard_max_group_size = 4;
  p->parallel_columns_scale_guard_min_groups = 128;
  p->enable_structure_specific_rules = 1;
  p->enable_two_row_variable_elimination = 1;
  p->two_row_variable_elimination_max_row_nnz = 8;
  p->two_row_variable_elimination_safety_tol = 1.0e-8;
  p->two_row_variable_elimination_min_candidates = 128;
  p->two_row_variable_elimination_min_candidate_ratio = 0.01;
  p->enable_zero_cost_product_variables = 1;
  p->zero_cost_product_variables_min_candidates = 128;
  p->zero_cost_product_variables_min_candidate_ratio = 0.01;
  p->enable_piecewise_linear_reformulation_variable_pair = 1;
  p->piecewise_linear_reformulation_variable_pair_epigraph_probe_pairs = 256;
  p->piecewise_linear_reformulation_variable_pair_epigraph_min_pairs = 4096;
  p->piecewise_linear_reformulation_variable_pair_epigraph_min_potential_gain = 0.20;
  p->piecewise_linear_reformulation_variable_pair_epigraph_min_actual_gain = 0.20;
  p->piecewise_linear_reformulation_variable_pair_epigraph_max_tail_cols = 8;
  p->piecewise_linear_reformulation_variable_pair_epigraph_max_quotient_terms_per_row = 5;
  p->piecewise_linear_reformulation_variable_pair_shifted_antipodal_probe_pairs = 256;
  p->piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs = 4096;
  p->piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_potential_gain = 0.20;
  p->piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_actual_gain = 0.20;
  p->piecewise_linear_reformulation_variable_pair_shifted_antipodal_max_quotient_terms_per_row = 6;
  p->enable_column_domination = 1;
  p->column_domination_probe_rows = 64;
  p->column_domination_probe_cols = 256;
  p->column_domination_probe_nnz = 256;
  p->column_domination_min_fixed_cols = 4096;
  p->column_domination_min_candidate_ratio = 0.20;
  p->enable_piecewise_linear_reformulation_absolute_value = 1;
  p->piecewise_linear_reformulation_absolute_value_residual_bound_mode = 0;
  p->piecewise_linear_reformulation_absolute_value_residual_bound_as_free_min = 1.0e8;
  p->enable_redundant_variable_bounds = 0;
  p->enable_startup = 1;
  p->bound_strengthening_bound_only_nnz_round_budget = 8000000;
}

int gpp_run_presolve(const gpp_lp* lp, const gpp_params* params, int keep_reduced_lp, gpp_summary* out) {
  return guarded([&] {
    if (!lp || !params || !out) throw std::invalid_argument("null argument");
    validate_lp(*lp);
    auto rec = std::make_unique<gpp_record>();
    const auto t0 = std::chrono::steady_clock::now();
    gpp::run_presolve(*lp, *params, rec->out);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (!keep_reduced_lp) {
      rec->out.reduced.free_owned();
      rec->out.reduced = gpp::WorkingLp{};
      rec->out.owns_reduced = false;
    }
    fill_summary(out, rec.get(), secs);
    rec.release();
  });
}

int gpp_preprocess(const gpp_lp* lp, const gpp_params* params, gpp_summary* out) {
  // folding::run_gpu_presolve_with_folding(lp, params, true, true) (folding.cu:172-213).
  return guarded([&] { preprocess_into(lp, params, out, true); });
}

int gpp_postsolve_device_lower(const double* x_red, const double* y_red, const double* z_red,
                               const gpp_summary* summary, const gpp_lp* original, const double* original_l,
                               double* x_org, double* y_org, double* z_org) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    const gpp_record* rec = summary->record;
    if (rec->folding.applied) throw std::invalid_argument("folded summaries postsolve through gpp_postprocess");
    gpp::run_postsolve(rec->out, x_red, y_red, z_red, original, x_org, y_org, z_org, original_l);
  });
}

int gpp_postsolve_device(const double* x_red, const double* y_red, const double* z_red, const gpp_summary* summary,
                         const gpp_lp* original, double* x_org, double* y_org, double* z_org) {
  return gpp_postsolve_device_lower(x_red, y_red, z_red, summary, original, nullptr, x_org, y_org, z_org);
}

int gpp_postprocess(const double* x_red, const double* y_red, const double* z_red, const gpp_summary* summary,
                    const gpp_lp* original, double* x_out, double* y_out, double* z_out) {
  // postsolve_and_unfold_to_host (folding.cu:215-261).
  return guarded([&] { postprocess_into(x_red, y_red, z_red, summary, original, x_out, y_out, z_out); });
}

void gpp_free_summary(gpp_summary* summary) {
  if (!summary || !summary->record) {
    if (summary) *summary = gpp_summary{};
    return;
  }
  gpp_record* rec = summary->record;
  try {
    rec->out.reduced.free_owned();
    gpp::free_folding(rec->folding);
    delete rec;
    gpp::ctx().sync("free summary");
  } catch (...) {
  }
  *summary = gpp_summary{};
}

int gpp_export_maps(const gpp_summary* summary, int32_t* row_red2org, int32_t* col_red2org) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    const gpp::Record& r = summary->record->out.record;
    auto s = gpp::ctx().stream;
    if (row_red2org && r.m) check(cudaMemcpyAsync(row_red2org, r.rows.p, 4 * size_t(r.m), cudaMemcpyDeviceToHost, s), "maps");
    if (col_red2org && r.n) check(cudaMemcpyAsync(col_red2org, r.cols.p, 4 * size_t(r.n), cudaMemcpyDeviceToHost, s), "maps");
    gpp::ctx().sync("export maps");
  });
}

int gpp_tape_sizes(const gpp_summary* summary, int64_t* records, int64_t* indices, int64_t* values, int64_t* fixed) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    const gpp::Record& r = summary->record->out.record;
    int64_t f = 0;
    for (const auto& seg : r.fixed) f += seg.count;
    if (records) *records = r.records;
    if (indices) *indices = r.indices;
    if (values) *values = r.values;
    if (fixed) *fixed = f;
  });
}

namespace {
void export_map(const gpp::FoldingResult& f, int32_t* row_color, int32_t* col_color, double* row_scale,
                double* col_scale) {
    if (!f.applied) return;
    auto s = gpp::ctx().stream;
    const size_t m = size_t(f.original_rows), n = size_t(f.original_cols);
    if (row_color && m) check(cudaMemcpyAsync(row_color, f.row_color.p, 4 * m, cudaMemcpyDeviceToHost, s), "fold map");
    if (col_color && n) check(cudaMemcpyAsync(col_color, f.col_color.p, 4 * n, cudaMemcpyDeviceToHost, s), "fold map");
    if (row_scale && m) check(cudaMemcpyAsync(row_scale, f.row_scale.p, 8 * m, cudaMemcpyDeviceToHost, s), "fold map");
    if (col_scale && n) check(cudaMemcpyAsync(col_scale, f.col_scale.p, 8 * n, cudaMemcpyDeviceToHost, s), "fold map");
    gpp::ctx().sync("export folding map");
}

const gpp::FoldingResult& run_result(const gpp_folding_run* run) {
  static const gpp::FoldingResult none{};
  if (!run) throw std::invalid_argument("null folding run");
  return run->handle ? *static_cast<const gpp::FoldingResult*>(run->handle) : none;
}
}  // namespace

int gpp_export_folding_map(const gpp_summary* summary, int32_t* row_color, int32_t* col_color, double* row_scale,
                           double* col_scale) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    export_map(summary->record->folding, row_color, col_color, row_scale, col_scale);
  });
}

int gpp_folding_run_export_map(const gpp_folding_run* run, int32_t* row_color, int32_t* col_color,
                               double* row_scale, double* col_scale) {
  return guarded([&] { export_map(run_result(run), row_color, col_color, row_scale, col_scale); });
}

int gpp_folding_run_unfold(const gpp_folding_run* run, const double* x_folded, const double* y_folded,
                           const double* z_folded, double* x_out, double* y_out, double* z_out) {
  return guarded([&] {
    const gpp::FoldingResult& f = run_result(run);
    if (!f.applied) throw std::invalid_argument("folding did not apply to this model");
    gpp::unfold_to_host(f, x_folded, y_folded, z_folded, x_out, y_out, z_out);
  });
}

int gpp_run_folding(const gpp_lp* lp, double tolerance, gpp_folding_run* out) {
  return guarded([&] {
    if (!lp || !out) throw std::invalid_argument("gpp_run_folding: null argument");
    *out = gpp_folding_run{};
    auto res = std::make_unique<gpp::FoldingResult>();
    out->original_rows = out->folded_rows = lp->A.rows;
    out->original_cols = out->folded_cols = lp->A.cols;
    const auto t0 = std::chrono::steady_clock::now();
    gpp::run_folding(*lp, tolerance, *res);
    gpp::ctx().sync("run_folding");
    out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (!res->applied) return;
    out->applied = 1;
    out->folded_rows = res->folded_rows;
    out->folded_cols = res->folded_cols;
    out->folded_lp = res->folded;
    out->owns_folded_lp = 1;
    out->row_color_id = res->row_color.p;
    out->col_color_id = res->col_color.p;
    out->row_scale = res->row_scale.p;
    out->col_scale = res->col_scale.p;
    out->handle = res.release();
  });
}

void gpp_free_folding_run(gpp_folding_run* run) {
  if (!run) return;
  auto* res = static_cast<gpp::FoldingResult*>(run->handle);
  if (res) {
    try {
      gpp::free_folding(*res);
    } catch (...) {
    }
    delete res;
  }
  *run = gpp_folding_run{};
}

int gpp_unfold_solution(const gpp_summary* summary, const double* x_folded, const double* y_folded,
                        const double* z_folded, double* x_out, double* y_out, double* z_out) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    const gpp::FoldingResult& f = summary->record->folding;
    if (!f.applied) throw std::invalid_argument("folding did not apply to this model");
    gpp::unfold_to_host(f, x_folded, y_folded, z_folded, x_out, y_out, z_out);
  });
}

int gpp_export_tape(const gpp_summary* summary, int32_t* types, int64_t* index_starts, int64_t* value_starts,
                    int32_t* indices, double* vals, int32_t* fixed_idx, double* fixed_val) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    const gpp::Record& r = summary->record->out.record;
    int64_t rk = 0, ik = 0, vk = 0;
    if (index_starts) index_starts[0] = 0;
    if (value_starts) value_starts[0] = 0;
    for (const auto& seg : r.segments) {
      auto t = gpp::to_host(seg.types.p, size_t(seg.count));
      auto is = gpp::to_host(seg.is.p, size_t(seg.count) + 1);
      auto vs = gpp::to_host(seg.vs.p, size_t(seg.count) + 1);
      auto id = gpp::to_host(seg.idx.p, size_t(seg.n_idx));
      auto v = gpp::to_host(seg.val.p, size_t(seg.n_val));
      for (int64_t k = 0; k < seg.count; ++k) {
        if (types) types[rk + k] = t[size_t(k)];
        if (index_starts) index_starts[rk + k + 1] = ik + is[size_t(k) + 1];
        if (value_starts) value_starts[rk + k + 1] = vk + vs[size_t(k) + 1];
      }
      if (indices) std::copy(id.begin(), id.end(), indices + ik);
      if (vals) std::copy(v.begin(), v.end(), vals + vk);
      rk += seg.count; ik += seg.n_idx; vk += seg.n_val;
    }
    int64_t fk = 0;
    for (const auto& seg : r.fixed) {
      auto a = gpp::to_host(seg.idx.p, size_t(seg.count));
      auto b = gpp::to_host(seg.val.p, size_t(seg.count));
      if (fixed_idx) std::copy(a.begin(), a.end(), fixed_idx + fk);
      if (fixed_val) std::copy(b.begin(), b.end(), fixed_val + fk);
      fk += seg.count;
    }
  });
}

int gpp_recovery_checkpoints(const gpp_summary* summary, int32_t* count, int32_t* kinds, int32_t* payloads,
                             int64_t* tape_positions) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    const gpp::Record& r = summary->record->out.record;
    if (count) *count = int32_t(r.timeline.size());
    for (size_t k = 0; k < r.timeline.size(); ++k) {
      if (kinds) kinds[k] = r.timeline[k].kind;
      if (payloads) payloads[k] = r.timeline[k].payload;
      if (tape_positions) tape_positions[k] = r.timeline[k].tape_position;
    }
  });
}

extern "C++" {
namespace {
const gpp::AbsValueRecovery& absolute_value_at(const gpp_summary* summary, int32_t index) {
  if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
  const auto& v = summary->record->out.record.absval;
  if (index < 0 || size_t(index) >= v.size()) throw std::invalid_argument("no absolute-value recovery at that index");
  return v[size_t(index)];
}
template <class T>
void copy_out(T* dst, const gpp::DBuf<T>& src, int64_t n) {
  if (dst && n > 0)
    check(cudaMemcpyAsync(dst, src.p, sizeof(T) * size_t(n), cudaMemcpyDeviceToHost, gpp::ctx().stream), "export");
}
template <class T>
void copy_in(gpp::DBuf<T>& dst, const T* src, int64_t n, const char* what) {
  if (n < 0) throw std::invalid_argument(std::string("negative count in ") + what);
  if (n > 0 && !src) throw std::invalid_argument(std::string("missing array ") + what);
  dst.alloc(size_t(n));
  if (n > 0)
    check(cudaMemcpyAsync(dst.p, src, sizeof(T) * size_t(n), cudaMemcpyHostToDevice, gpp::ctx().stream), what);
}
}  // namespace
}

int gpp_absolute_value_sizes(const gpp_summary* summary, int32_t index, int32_t sizes[6]) {
  return guarded([&] {
    const auto& a = absolute_value_at(summary, index);
    if (!sizes) throw std::invalid_argument("sizes is null");
    sizes[0] = a.pattern;
    sizes[1] = a.splits;
    sizes[2] = a.pairs;
    sizes[3] = a.links;
    sizes[4] = a.max_groups;
    sizes[5] = a.max_entries;
  });
}

int gpp_export_absolute_value(const gpp_summary* summary, int32_t index, int32_t* split_t, int32_t* split_e,
                              double* split_rho, int32_t* pair_bound, int32_t* pair_free, int32_t* linked_slack,
                              int32_t* linked_t, double* linked_factor, int32_t* max_slack, int32_t* max_starts,
                              int32_t* max_t, double* max_factor) {
  return guarded([&] {
    const auto& a = absolute_value_at(summary, index);
    copy_out(split_t, a.split_t, a.splits);
    copy_out(split_e, a.split_e, a.splits);
    copy_out(split_rho, a.split_rho, a.splits);
    copy_out(pair_bound, a.pair_bound, a.pairs);
    copy_out(pair_free, a.pair_free, a.pairs);
    copy_out(linked_slack, a.link_slack, a.links);
    copy_out(linked_t, a.link_t, a.links);
    copy_out(linked_factor, a.link_factor, a.links);
    copy_out(max_slack, a.max_slack, a.max_groups);
    copy_out(max_starts, a.max_start, a.max_groups ? a.max_groups + 1 : 0);
    copy_out(max_t, a.max_t, a.max_entries);
    copy_out(max_factor, a.max_factor, a.max_entries);
    if (max_starts && !a.max_groups) max_starts[0] = 0;
    gpp::ctx().sync("export absolute-value recovery");
  });
}

int gpp_variable_pair_size(const gpp_summary* summary, int32_t index, int32_t* count) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    const auto& v = summary->record->out.record.varpair;
    if (index < 0 || size_t(index) >= v.size()) throw std::invalid_argument("no variable-pair recovery at that index");
    if (!count) throw std::invalid_argument("count is null");
    *count = v[size_t(index)].count;
  });
}

int gpp_export_variable_pair(const gpp_summary* summary, int32_t index, int32_t* plus_cols, int32_t* minus_cols,
                             int32_t* root_plus_cols, int32_t* root_minus_cols, double* plus_shift,
                             double* minus_shift) {
  return guarded([&] {
    if (!summary || !summary->record) throw std::invalid_argument("summary has no recovery record");
    const auto& v = summary->record->out.record.varpair;
    if (index < 0 || size_t(index) >= v.size()) throw std::invalid_argument("no variable-pair recovery at that index");
    const auto& r = v[size_t(index)];
    copy_out(plus_cols, r.plus, r.count);
    copy_out(minus_cols, r.minus, r.count);
    copy_out(root_plus_cols, r.root_plus, r.count);
    copy_out(root_minus_cols, r.root_minus, r.count);
    copy_out(plus_shift, r.plus_shift, r.count);
    copy_out(minus_shift, r.minus_shift, r.count);
    gpp::ctx().sync("export variable-pair recovery");
  });
}

int gpp_restore_absolute_value(double* x_org, const gpp_absolute_value_recovery* steps, int32_t count,
                               const double* original_l) {
  return guarded([&] {
    if (count < 0 || (count > 0 && (!steps || !x_org))) throw std::invalid_argument("invalid recovery steps");
    for (int32_t k = count - 1; k >= 0; --k) {
      const gpp_absolute_value_recovery& h = steps[k];
      gpp::AbsValueRecovery d;
      d.pattern = h.pattern;
      d.splits = h.split_count;
      d.pairs = h.pair_count;
      d.links = h.linked_count;
      d.max_groups = h.max_group_count;
      if (d.max_groups < 0) throw std::invalid_argument("negative max-slack group count");
      if (d.max_groups > 0 && !h.max_starts) throw std::invalid_argument("missing array max_starts");
      d.max_entries = d.max_groups ? h.max_starts[d.max_groups] : 0;
      for (int32_t g = 0; g < d.max_groups; ++g)
        if (h.max_starts[g] < 0 || h.max_starts[g] > h.max_starts[g + 1])
          throw std::invalid_argument("max_starts is not ascending");
      auto ids_ok = [](const int32_t* v, int32_t n) {
        for (int32_t i = 0; i < n; ++i)
          if (v[i] < 0) return false;
        return true;
      };
      copy_in(d.split_t, h.split_t, d.splits, "split_t");
      copy_in(d.split_e, h.split_e, d.splits, "split_e");
      copy_in(d.split_rho, h.split_rho, d.splits, "split_rho");
      copy_in(d.pair_bound, h.pair_bound, d.pairs, "pair_bound");
      copy_in(d.pair_free, h.pair_free, d.pairs, "pair_free");
      copy_in(d.link_slack, h.linked_slack, d.links, "linked_slack");
      copy_in(d.link_t, h.linked_t, d.links, "linked_t");
      copy_in(d.link_factor, h.linked_factor, d.links, "linked_factor");
      copy_in(d.max_slack, h.max_slack, d.max_groups, "max_slack");
      copy_in(d.max_start, h.max_starts, d.max_groups ? d.max_groups + 1 : 0, "max_starts");
      copy_in(d.max_t, h.max_t, d.max_entries, "max_t");
      copy_in(d.max_factor, h.max_factor, d.max_entries, "max_factor");
      if (!ids_ok(h.split_t, d.splits) || !ids_ok(h.split_e, d.splits) || !ids_ok(h.pair_bound, d.pairs) ||
          !ids_ok(h.pair_free, d.pairs) || !ids_ok(h.linked_slack, d.links) || !ids_ok(h.linked_t, d.links) ||
          !ids_ok(h.max_slack, d.max_groups) || !ids_ok(h.max_t, d.max_entries))
        throw std::invalid_argument("negative column id in a recovery step");
      gpp::restore_absolute_value(x_org, d, original_l, gpp::ctx().stream);
    }
    gpp::ctx().sync("restore absolute value");
  });
}

int gpp_row_activity_summary(const gpp_csr* A, const double* l, const double* u, double zero_tol,
                             const uint8_t* keep_row, const uint8_t* keep_col, const int32_t* live_degrees,
                             double* min_fin, double* max_fin, int32_t* min_inf, int32_t* max_inf) {
  return guarded([&] {
    gpp::DevCsr M{A->rows, A->cols, A->nnz, A->rowPtr, A->colVal, A->nzVal};
    gpp::invalidate_schedules();
    gpp::row_activity_summary(M, l, u, zero_tol, keep_row, keep_col, live_degrees, min_fin, max_fin, min_inf,
                              max_inf, gpp::ctx().stream);
    gpp::ctx().sync("activity summary");
  });
}

int gpp_live_stats(const gpp_csr* M, const uint8_t* keep_outer, const uint8_t* keep_inner, int32_t* degree,
                   uint8_t* empty, uint8_t* singleton, int32_t* support, double* coefficient,
                   unsigned long long* total) {
  return guarded([&] {
    gpp::DevCsr D{M->rows, M->cols, M->nnz, M->rowPtr, M->colVal, M->nzVal};
    gpp::invalidate_schedules();
    if (total) check(cudaMemsetAsync(total, 0, sizeof(*total), gpp::ctx().stream), "total");
    gpp::live_stats_side(D, keep_outer, keep_inner, degree, empty, singleton, support, coefficient, total,
                         gpp::ctx().stream);
    gpp::ctx().sync("live stats");
  });
}

int gpp_col_max_abs(const gpp_csr* AT, const uint8_t* keep_row, double* out) {
  return guarded([&] {
    gpp::DevCsr D{AT->rows, AT->cols, AT->nnz, AT->rowPtr, AT->colVal, AT->nzVal};
    gpp::invalidate_schedules();
    gpp::col_max_abs(D, keep_row, out, gpp::ctx().stream);
    gpp::ctx().sync("col max");
  });
}

int gpp_compact_and_transpose(const gpp_csr* A, const uint8_t* keep_row, const uint8_t* keep_col, gpp_csr* A_out,
                              gpp_csr* AT_out) {
  return guarded([&] {
    auto s = gpp::ctx().stream;
    gpp::DevCsr D{A->rows, A->cols, A->nnz, A->rowPtr, A->colVal, A->nzVal};
    gpp::invalidate_schedules();
    gpp::DBuf<int32_t> rmap(size_t(std::max(D.rows, 1)), s), cmap(size_t(std::max(D.cols, 1)), s);
    const int m_new = gpp::build_old_to_new(keep_row, D.rows, rmap.p, s);
    const int n_new = gpp::build_old_to_new(keep_col, D.cols, cmap.p, s);
    gpp::DevCsr C = gpp::compact_csr(D, rmap.p, m_new, cmap.p, n_new, s);
    gpp::DevCsr T = gpp::transpose_csr(C, s);
    gpp::ctx().sync("compact and transpose");
    *A_out = gpp_csr{C.rows, C.cols, C.nnz, C.ptr, C.idx, C.val};
    *AT_out = gpp_csr{T.rows, T.cols, T.nnz, T.ptr, T.idx, T.val};
  });
}

int gpp_parallel_row_hashes(const gpp_csr* A, const uint8_t* keep_row, const uint8_t* keep_col, int mode,
                            uint64_t* hashes) {
  return guarded([&] {
    gpp::DevCsr D{A->rows, A->cols, A->nnz, A->rowPtr, A->colVal, A->nzVal};
    gpp::invalidate_schedules();
    gpp::parallel_row_hashes(D, keep_row, keep_col, mode, hashes, gpp::ctx().stream);
    gpp::ctx().sync("row hashes");
  });
}

int gpp_sort_pairs(uint64_t* keys, int32_t* values, int64_t n) {
  return guarded([&] {
    gpp::radix_sort_pairs(keys, values, n, gpp::ctx().stream);
    gpp::ctx().sync("sort pairs");
  });
}

int gpp_sort_pairs_static(uint64_t* keys, int32_t* values, int64_t n, void* stream) {
  return guarded([&] { gpp::radix_sort_pairs_static(keys, values, n, static_cast<cudaStream_t>(stream)); });
}

void gpp_inject_alloc_failure(int64_t after) { gpp::inject_alloc_failure(after); }

int gpp_device_alloc(void** ptr, size_t bytes) {
  return guarded([&] {
    if (!ptr) throw std::invalid_argument("null argument");
    *ptr = nullptr;
    if (bytes) check(cudaMalloc(ptr, bytes), "cudaMalloc");
  });
}

void gpp_device_free(void* p) {
  if (!p) return;
  try {
    cudaFreeAsync(p, gpp::ctx().stream);
    gpp::ctx().sync("device free");
  } catch (...) {
  }
}

const char* gpp_last_error(void) { return gpp::last_error(); }

void gpp_profile_enable(int enable) { gpp::profile_enable(enable != 0); }

int gpp_profile_read(int index, char* name, size_t name_len, int64_t* launches, double* ms, double* bytes) {
  try {
    static thread_local std::vector<gpp::ProfileSummary> cache;
    if (index == 0) cache = gpp::profile_summary();
    if (index >= 0 && size_t(index) < cache.size()) {
      const auto& e = cache[size_t(index)];
      if (name && name_len) {
        std::strncpy(name, e.name.c_str(), name_len - 1);
        name[name_len - 1] = 0;
      }
      if (launches) *launches = e.launches;
      if (ms) *ms = e.ms;
      if (bytes) *bytes = e.bytes;
    }
    return int(cache.size());
  } catch (const std::exception& e) {
    gpp::set_last_error(e.what());
    return -1;
  }
}

uint64_t gpp_kernel_launches(int reset) {
  const uint64_t v = gpp::launch_counter();
  if (reset) gpp::launch_counter() = 0;
  return v;
}

uint64_t gpp_host_syncs(int reset) {
  const uint64_t v = gpp::sync_counter();
  if (reset) gpp::sync_counter() = 0;
  return v;
}


int gpp_preprocess_batch(const gpp_lp* lps, int32_t count, const gpp_params* params, int32_t workers,
                         gpp_summary* out, int32_t* status) {
  if (count < 0 || (count > 0 && (!lps || !params || !out))) {
    gpp::set_last_error("gpp_preprocess_batch: null argument or negative count");
    return GPP_ERR_INVALID;
  }
  if (count == 0) return GPP_OK;
  const int w = workers > 0 ? workers : kDefaultBatchWorkers;
  return guarded([&] {
    check(cudaDeviceSynchronize(), "before batch");   // inputs queued on any stream are complete
    for (int32_t k = 0; k < count; ++k) out[k] = gpp_summary{};
    const int rc = run_batch(count, w, largest_first(lps, count), status,
                             [&](int k) { preprocess_into(&lps[k], params, &out[k], false); });
    if (rc != GPP_OK) throw BatchFailure{rc};
  });
}

int gpp_postprocess_batch(const double* const* x_red, const double* const* y_red, const double* const* z_red,
                          const gpp_summary* summaries, const gpp_lp* originals, int32_t count, int32_t workers,
                          double* const* x_out, double* const* y_out, double* const* z_out, int32_t* status) {
  if (count < 0 || (count > 0 && (!summaries || !originals))) {
    gpp::set_last_error("gpp_postprocess_batch: null argument or negative count");
    return GPP_ERR_INVALID;
  }
  if (count == 0) return GPP_OK;
  const int w = workers > 0 ? workers : kDefaultBatchWorkers;
  auto at = [](auto a, int k) { return a ? a[k] : nullptr; };
  return guarded([&] {
    check(cudaDeviceSynchronize(), "before batch");
    const int rc = run_batch(count, w, largest_first(originals, count), status, [&](int k) {
      postprocess_into(at(x_red, k), at(y_red, k), at(z_red, k), &summaries[k], &originals[k], at(x_out, k),
                       at(y_out, k), at(z_out, k));
    });
    if (rc != GPP_OK) throw BatchFailure{rc};
  });
}

int gpp_batch_autotune(const gpp_lp* lps, int32_t count, const gpp_params* params, int32_t max_workers,
                       int32_t* best_workers, double* rates) {
  if (count <= 0 || !lps || !params || !best_workers || max_workers < 1) {
    gpp::set_last_error("gpp_batch_autotune: empty batch, null argument or max_workers < 1");
    return GPP_ERR_INVALID;
  }
  return guarded([&] {
    // A sample that keeps the batch's size mix: every k-th LP of the
    // largest-first order, at most kAutotuneSample of them.
    const std::vector<int> order = largest_first(lps, count);
    const int stride = std::max<int>(1, (count + kAutotuneSample - 1) / kAutotuneSample);
    std::vector<gpp_lp> sample;
    for (size_t i = 0; i < order.size(); i += size_t(stride)) sample.push_back(lps[order[i]]);
    std::vector<gpp_summary> out(sample.size());
    double best_rate = -1.0;
    int best = 1, tried = 0;
    for (int w = 1; w <= max_workers; w *= 2) {
      check(cudaDeviceSynchronize(), "autotune");
      const auto t0 = std::chrono::steady_clock::now();
      const int rc = gpp_preprocess_batch(sample.data(), int32_t(sample.size()), params, w, out.data(), nullptr);
      const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      for (auto& o : out) gpp_free_summary(&o);
      if (rc != GPP_OK) throw BatchFailure{rc};
      const double rate = double(sample.size()) / std::max(secs, 1e-9);
      if (rates) rates[tried] = rate;
      ++tried;
      // A larger pool must beat the best so far by 5% to be chosen.
      if (rate > best_rate * 1.05) { best_rate = rate; best = w; }
    }
    *best_workers = best;
  });
}

int gpp_preprocess_traced(const gpp_lp* lp, const gpp_params* params, gpp_summary* out, float* features,
                          int32_t* round_info, int64_t* round_nnz, int32_t max_rounds, int32_t* rounds) {
  return guarded([&] {
    if (!rounds || max_rounds < 0) throw std::invalid_argument("gpp_preprocess_traced: bad round buffer");
    std::vector<gpp::RoundRecord> trace;
    preprocess_into(lp, params, out, true, nullptr, &trace);
    *rounds = int32_t(trace.size());
    for (size_t r = 0; r < trace.size() && int32_t(r) < max_rounds; ++r) {
      const auto& t = trace[r];
      if (features) std::copy(t.features, t.features + gpp::kScheduleFeatures, features + r * gpp::kScheduleFeatures);
      if (round_info) {
        round_info[4 * r + 0] = t.phase;
        round_info[4 * r + 1] = t.iteration;
        round_info[4 * r + 2] = int32_t(t.ran);
        round_info[4 * r + 3] = int32_t(t.changed);
      }
      if (round_nnz) {
        round_nnz[2 * r + 0] = t.nnz_before;
        round_nnz[2 * r + 1] = t.nnz_after;
      }
    }
  });
}

int gpp_schedule_model_create_per_rule(const float* params, const double* skip_below, double stop_above,
                                       gpp_schedule_model** out) {
  return guarded([&] {
    if (!params || !out || !skip_below || !(stop_above >= 0.0))
      throw std::invalid_argument("gpp_schedule_model_create: null argument or threshold out of range");
    for (int g = 0; g < gpp::kGatedRules; ++g)
      if (!(skip_below[g] >= 0.0 && skip_below[g] <= 1.0))
        throw std::invalid_argument("gpp_schedule_model_create: skip threshold out of range");
    auto m = std::make_unique<gpp_schedule_model>();
    m->policy = std::make_unique<gpp::MlpSchedule>(params, skip_below, stop_above);
    *out = m.release();
  });
}

int gpp_schedule_model_create(const float* params, double skip_below, double stop_above,
                              gpp_schedule_model** out) {
  double each[gpp::kGatedRules];
  std::fill(each, each + gpp::kGatedRules, skip_below);
  return gpp_schedule_model_create_per_rule(params, each, stop_above, out);
}

void gpp_schedule_model_free(gpp_schedule_model* model) { delete model; }

int gpp_preprocess_scheduled(const gpp_lp* lp, const gpp_params* params, gpp_schedule_model* model,
                             gpp_summary* out) {
  return guarded([&] {
    if (!model) throw std::invalid_argument("gpp_preprocess_scheduled: null model");
    preprocess_into(lp, params, out, true, model->policy.get(), nullptr);
  });
}

int gpp_mlp_train(float* params, const float* X, const float* Y, const float* M, int64_t n, int32_t epochs,
                  int32_t batch, float lr, uint64_t seed, float* loss_per_epoch) {
  return guarded([&] {
    if (!params || !X || !Y || !M) throw std::invalid_argument("gpp_mlp_train: null argument");
    gpp::mlp_train(params, X, Y, M, n, epochs, batch, lr, seed, loss_per_epoch);
  });
}

int gpp_mlp_forward(const float* params, const float* X, int64_t n, float* probs) {
  return guarded([&] {
    if (!params || (n > 0 && (!X || !probs))) throw std::invalid_argument("gpp_mlp_forward: null argument");
    gpp::mlp_forward(params, X, n, probs);
  });
}

int gpp_mlp_gradients(const float* params, const float* X, const float* Y, const float* M, int64_t n, float* grads,
                      float* loss) {
  return guarded([&] {
    if (!params || !X || !Y || !M || !grads) throw std::invalid_argument("gpp_mlp_gradients: null argument");
    gpp::mlp_gradients(params, X, Y, M, n, grads, loss);
  });
}

int gpp_mps_read(const char* path, gpp_mps_model** out) {
  try {
    if (!path || !out) throw std::invalid_argument("gpp_mps_read: null argument");
    auto m = std::make_unique<gpp_mps_model>();
    m->m = gpp::read_mps_file(path);
    *out = m.release();
    gpp::set_last_error("");
    return GPP_OK;
  } catch (const std::invalid_argument& e) {
    gpp::set_last_error(e.what());
    return GPP_ERR_INVALID;
  } catch (const std::exception& e) {
    gpp::set_last_error(e.what());
    return GPP_ERR_RUNTIME;
  }
}

int gpp_mps_read_string(const char* text, gpp_mps_model** out) {
  try {
    if (!text || !out) throw std::invalid_argument("gpp_mps_read_string: null argument");
    auto m = std::make_unique<gpp_mps_model>();
    m->m = gpp::read_mps_text(text);
    *out = m.release();
    gpp::set_last_error("");
    return GPP_OK;
  } catch (const std::invalid_argument& e) {
    gpp::set_last_error(e.what());
    return GPP_ERR_INVALID;
  } catch (const std::exception& e) {
    gpp::set_last_error(e.what());
    return GPP_ERR_RUNTIME;
  }
}

int gpp_mps_info(const gpp_mps_model* model, int32_t* rows, int32_t* cols, int64_t* nnz, double* obj_constant,
                 char* name, size_t name_len) {
  if (!model) return GPP_ERR_INVALID;
  const gpp::MpsModel& m = model->m;
  if (rows) *rows = m.rows;
  if (cols) *cols = m.cols;
  if (nnz) *nnz = int64_t(m.csr_val.size());
  if (obj_constant) *obj_constant = m.obj_constant;
  if (name && name_len) {
    const size_t k = std::min(name_len - 1, m.name.size());
    std::memcpy(name, m.name.data(), k);
    name[k] = '\0';
  }
  return GPP_OK;
}

int gpp_mps_arrays(const gpp_mps_model* model, int64_t* row_ptr, int32_t* col_idx, double* csr_val, int64_t* col_ptr,
                   int32_t* row_idx, double* csc_val, double* c, double* AL, double* AU, double* l, double* u) {
  if (!model) return GPP_ERR_INVALID;
  const gpp::MpsModel& m = model->m;
  auto put = [](auto* dst, const auto& v) { if (dst) std::copy(v.begin(), v.end(), dst); };
  put(row_ptr, m.row_ptr); put(col_idx, m.col_idx); put(csr_val, m.csr_val);
  put(col_ptr, m.col_ptr); put(row_idx, m.row_idx); put(csc_val, m.csc_val);
  put(c, m.cost); put(AL, m.row_lower); put(AU, m.row_upper); put(l, m.col_lower); put(u, m.col_upper);
  return GPP_OK;
}

void gpp_mps_free(gpp_mps_model* model) { delete model; }

int gpp_mps_upload(const gpp_mps_model* model, gpp_lp* out) {
  return guarded([&] {
    if (!model || !out) throw std::invalid_argument("gpp_mps_upload: null argument");
    const gpp::MpsModel& m = model->m;
    const int64_t nnz = int64_t(m.csr_val.size());
    if (nnz > int64_t(INT32_MAX)) throw std::length_error("nnz exceeds the 32-bit offset range of this build");
    *out = gpp_lp{};
    auto up = [](const auto& v, auto** dst) {
      using T = std::remove_pointer_t<std::remove_reference_t<decltype(*dst)>>;
      check(cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * std::max<size_t>(v.size(), 1)), "cudaMalloc");
      if (!v.empty()) check(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
    };
    try {
      const std::vector<gpp_offset> rp(m.row_ptr.begin(), m.row_ptr.end()), cp(m.col_ptr.begin(), m.col_ptr.end());
      out->A = {m.rows, m.cols, gpp_offset(nnz), nullptr, nullptr, nullptr};
      out->AT = {m.cols, m.rows, gpp_offset(nnz), nullptr, nullptr, nullptr};
      up(rp, &out->A.rowPtr); up(m.col_idx, &out->A.colVal); up(m.csr_val, &out->A.nzVal);
      up(cp, &out->AT.rowPtr); up(m.row_idx, &out->AT.colVal); up(m.csc_val, &out->AT.nzVal);
      up(m.cost, &out->c); up(m.row_lower, &out->AL); up(m.row_upper, &out->AU);
      up(m.col_lower, &out->l); up(m.col_upper, &out->u);
      out->obj_constant = m.obj_constant;
    } catch (...) {
      gpp_lp_free(out);
      throw;
    }
  });
}

int gpp_lp_from_host(const gpp_host_lp* host, gpp_lp* dev) {
  return guarded([&] {
    if (!host || !dev) throw std::invalid_argument("gpp_lp_from_host: null argument");
    const int32_t m = host->rows, n = host->cols;
    const gpp_offset nnz = host->nnz;
    if (m < 0 || n < 0 || nnz < 0) throw std::invalid_argument("gpp_lp_from_host: negative LP dimensions");
    if (!host->row_ptr || (nnz > 0 && (!host->col_idx || !host->val)) ||
        (n > 0 && (!host->c || !host->l || !host->u)) || (m > 0 && (!host->AL || !host->AU)))
      throw std::invalid_argument("gpp_lp_from_host: host array missing");
    if (!dev->A.rowPtr || !dev->AT.rowPtr || (nnz > 0 && (!dev->A.colVal || !dev->A.nzVal || !dev->AT.colVal ||
                                                          !dev->AT.nzVal)) ||
        (n > 0 && (!dev->c || !dev->l || !dev->u)) || (m > 0 && (!dev->AL || !dev->AU)))
      throw std::invalid_argument("gpp_lp_from_host: device array missing");
    auto& c = gpp::ctx();
    const cudaStream_t s = c.stream, side = c.side_stream();
    auto up = [](void* d, const void* h, size_t bytes, cudaStream_t st) {
      if (bytes) check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st), "gpp_lp_from_host: upload");
    };
    up(dev->A.rowPtr, host->row_ptr, sizeof(gpp_offset) * (size_t(m) + 1), s);
    up(dev->A.colVal, host->col_idx, sizeof(int32_t) * size_t(nnz), s);
    up(dev->A.nzVal, host->val, sizeof(double) * size_t(nnz), s);
    // The vectors follow A on the side stream, so they cross the bus while
    // the engine stream checks and transposes A.
    cudaEvent_t a_done = nullptr, vec_done = nullptr;
    check(cudaEventCreateWithFlags(&a_done, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&vec_done, cudaEventDisableTiming), "cudaEventCreate");
    // On every exit, error paths included, the side stream's copies are
    // finished before the caller gets its host arrays back.
    struct Events {
      cudaEvent_t a, b;
      cudaStream_t side;
      ~Events() {
        cudaStreamSynchronize(side);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
      }
    } events{a_done, vec_done, side};
    check(cudaEventRecord(a_done, s), "cudaEventRecord");
    check(cudaStreamWaitEvent(side, a_done, 0), "cudaStreamWaitEvent");
    up(dev->c, host->c, sizeof(double) * size_t(n), side);
    up(dev->l, host->l, sizeof(double) * size_t(n), side);
    up(dev->u, host->u, sizeof(double) * size_t(n), side);
    up(dev->AL, host->AL, sizeof(double) * size_t(m), side);
    up(dev->AU, host->AU, sizeof(double) * size_t(m), side);
    check(cudaEventRecord(vec_done, side), "cudaEventRecord");
    const gpp::DevCsr A{m, n, nnz, dev->A.rowPtr, dev->A.colVal, dev->A.nzVal};
    const gpp::DevCsr AT{n, m, nnz, dev->AT.rowPtr, dev->AT.colVal, dev->AT.nzVal};
    const bool valid = gpp::csr_structure_valid(A, s);
    if (valid) gpp::transpose_csr_into(A, AT, s);
    check(cudaStreamWaitEvent(s, vec_done, 0), "cudaStreamWaitEvent");
    c.sync("gpp_lp_from_host");
    if (!valid)
      throw std::invalid_argument("gpp_lp_from_host: A is not a valid CSR (row pointers or column indices)");
    dev->A.rows = m;
    dev->A.cols = n;
    dev->A.nnz = nnz;
    dev->AT.rows = n;
    dev->AT.cols = m;
    dev->AT.nnz = nnz;
    dev->obj_constant = host->obj_constant;
  });
}

void gpp_lp_free(gpp_lp* lp) {
  if (!lp) return;
  for (void* p : {static_cast<void*>(lp->A.rowPtr), static_cast<void*>(lp->A.colVal), static_cast<void*>(lp->A.nzVal),
                  static_cast<void*>(lp->AT.rowPtr), static_cast<void*>(lp->AT.colVal),
                  static_cast<void*>(lp->AT.nzVal), static_cast<void*>(lp->c), static_cast<void*>(lp->AL),
                  static_cast<void*>(lp->AU), static_cast<void*>(lp->l), static_cast<void*>(lp->u)})
    if (p) cudaFree(p);
  *lp = gpp_lp{};
}

namespace {
void require_reduced(const gpp_summary* summary, const char* who) {
  if (!summary || !summary->record) throw std::invalid_argument(std::string(who) + ": null argument");
  if (summary->has_infeasible || summary->has_unbounded)
    throw std::invalid_argument(std::string(who) + ": presolve ended infeasible or unbounded; no reduced LP");
}
}  // namespace

int gpp_reduced_to_device(const gpp_summary* summary, gpp_lp* out) {
  return guarded([&] {
    require_reduced(summary, "gpp_reduced_to_device");
    if (!out) throw std::invalid_argument("gpp_reduced_to_device: null argument");
    const gpp_lp& r = summary->reduced_lp;
    if (r.A.rows <= 0 || r.A.cols <= 0 || r.A.nnz <= 0)
      throw std::invalid_argument("gpp_reduced_to_device: the reduced LP is empty");
    *out = gpp_lp{};
    auto dup = [](const auto* src, size_t count, auto** dst) {
      using T = std::remove_const_t<std::remove_pointer_t<decltype(src)>>;
      check(cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * std::max<size_t>(count, 1)), "cudaMalloc");
      if (count) check(cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyDeviceToDevice), "handoff copy");
    };
    try {
      const size_t m = size_t(r.A.rows), n = size_t(r.A.cols), nnz = size_t(r.A.nnz);
      out->A = {r.A.rows, r.A.cols, r.A.nnz, nullptr, nullptr, nullptr};
      out->AT = {r.AT.rows, r.AT.cols, r.AT.nnz, nullptr, nullptr, nullptr};
      dup(r.A.rowPtr, m + 1, &out->A.rowPtr); dup(r.A.colVal, nnz, &out->A.colVal);
      dup(r.A.nzVal, nnz, &out->A.nzVal);
      dup(r.AT.rowPtr, n + 1, &out->AT.rowPtr); dup(r.AT.colVal, nnz, &out->AT.colVal);
      dup(r.AT.nzVal, nnz, &out->AT.nzVal);
      dup(r.c, n, &out->c); dup(r.AL, m, &out->AL); dup(r.AU, m, &out->AU);
      dup(r.l, n, &out->l); dup(r.u, n, &out->u);
      out->obj_constant = r.obj_constant;
    } catch (...) {
      gpp_lp_free(out);
      throw;
    }
  });
}

int gpp_reduced_to_host(const gpp_summary* summary, gpp_offset* row_ptr, int32_t* col_idx, double* val, double* c,
                        double* AL, double* AU, double* l, double* u, double* obj_constant) {
  return guarded([&] {
    require_reduced(summary, "gpp_reduced_to_host");
    const gpp_lp& r = summary->reduced_lp;
    const size_t m = size_t(std::max(0, r.A.rows)), n = size_t(std::max(0, r.A.cols)),
                 nnz = size_t(std::max<gpp_offset>(0, r.A.nnz));
    auto get = [](void* dst, const void* src, size_t bytes) {
      if (dst && bytes) check(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost), "handoff copy");
    };
    if (row_ptr && !r.A.rowPtr) {
      for (size_t i = 0; i <= m; ++i) row_ptr[i] = 0;
    } else {
      get(row_ptr, r.A.rowPtr, sizeof(gpp_offset) * (m + 1));
    }
    get(col_idx, r.A.colVal, sizeof(int32_t) * nnz);
    get(val, r.A.nzVal, sizeof(double) * nnz);
    get(c, r.c, sizeof(double) * n);
    get(AL, r.AL, sizeof(double) * m);
    get(AU, r.AU, sizeof(double) * m);
    get(l, r.l, sizeof(double) * n);
    get(u, r.u, sizeof(double) * n);
    if (obj_constant) *obj_constant = r.obj_constant;
  });
}

int gpp_export_reduced(const gpp_summary* summary, const char* out_dir, const char* model_name) {
  return guarded([&] {
    if (!summary || !summary->record || !out_dir) throw std::invalid_argument("gpp_export_reduced: null argument");
    namespace fs = std::filesystem;
    const fs::path dir(out_dir);
    fs::create_directories(dir);
    const gpp_lp& lp = summary->reduced_lp;
    std::ofstream meta(dir / "meta.txt");
    if (!meta) throw std::runtime_error("failed to open export meta");
    meta << std::setprecision(17);
    meta << "format gpu_preprocessor_reduced_lp_v1\noffset_bits 32\n";
    meta << "model " << (model_name ? model_name : "") << "\n";
    meta << "status " << (summary->has_infeasible ? "infeasible" : summary->has_unbounded ? "unbounded" : "ok") << "\n";
    meta << "original_rows " << summary->original_rows << "\noriginal_cols " << summary->original_cols << "\n";
    meta << "folding_applied " << int(summary->folding_applied) << "\nfolded_rows " << summary->folded_rows
         << "\nfolded_cols " << summary->folded_cols << "\n";
    meta << "reduced_rows " << summary->reduced_rows << "\nreduced_cols " << summary->reduced_cols
         << "\nreduced_nnz " << summary->reduced_nnz << "\n";
    meta << "obj_constant " << lp.obj_constant << "\nobjective_shift " << summary->obj_constant_delta << "\n";
    meta << "preprocessing_seconds " << summary->preprocessing_seconds << "\npresolve_seconds "
         << summary->elapsed_seconds << "\n";
    meta << "iterations " << summary->iterations << "\n";
    if (!meta) throw std::runtime_error("failed to write export meta");
    auto write = [&](const char* name, const void* dev, size_t bytes) {
      std::vector<char> host(bytes);
      if (bytes) check(cudaMemcpy(host.data(), dev, bytes, cudaMemcpyDeviceToHost), "export copy");
      std::ofstream f(dir / name, std::ios::binary);
      f.write(host.data(), std::streamsize(bytes));
      if (!f) throw std::runtime_error(std::string("failed to write ") + name);
    };
    const size_t m = size_t(lp.A.rows), n = size_t(lp.A.cols), nnz = size_t(lp.A.nnz);
    if (m == 0) {
      const int32_t zero = 0;
      std::ofstream f(dir / "A_rowPtr_i32.bin", std::ios::binary);
      f.write(reinterpret_cast<const char*>(&zero), sizeof(zero));
    } else {
      write("A_rowPtr_i32.bin", lp.A.rowPtr, sizeof(gpp_offset) * (m + 1));
    }
    write("A_colVal_i32.bin", lp.A.colVal, sizeof(int32_t) * nnz);
    write("A_nzVal_f64.bin", lp.A.nzVal, sizeof(double) * nnz);
    write("c_f64.bin", lp.c, sizeof(double) * n);
    write("l_f64.bin", lp.l, sizeof(double) * n);
    write("u_f64.bin", lp.u, sizeof(double) * n);
    write("AL_f64.bin", lp.AL, sizeof(double) * m);
    write("AU_f64.bin", lp.AU, sizeof(double) * m);
  });
}
}  // extern "C"
