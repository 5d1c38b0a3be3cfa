// Symmetry folding.  Colour refinement is not built yet: a call with folding
// enabled fails loudly instead of silently skipping the reduction.
#include "folding.hpp"

namespace gpp {

void run_folding(const gpp_lp& lp, double tolerance, FoldingResult& out) {
  if (!std::isfinite(tolerance) || tolerance < 0.0)
    throw std::invalid_argument("folding tolerance must be finite and nonnegative");
  out.original_rows = out.folded_rows = lp.A.rows;
  out.original_cols = out.folded_cols = lp.A.cols;
  if (lp.A.rows == 0 || lp.A.cols == 0) return;
  throw std::runtime_error("folding is not available in this build; call with enable_folding = 0");
}

void free_folding(FoldingResult& f) { f = FoldingResult{}; }

void unfold_to_host(const FoldingResult&, const double*, const double*, const double*, double*, double*, double*) {
  throw std::runtime_error("folding is not available in this build");
}

}  // namespace gpp
