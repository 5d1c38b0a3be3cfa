// Rules whose CUDA restatement is not built yet fail loudly, so a run with
// them enabled can never silently skip a reduction.
#include "folding.hpp"

namespace gpp {

#define GPP_PENDING(name, ...) \
  void name(__VA_ARGS__) { throw std::runtime_error(#name " is not available in this build; disable it in gpp_params"); }
GPP_PENDING(rule_doubleton_equations, Plan&, const WorkingLp&, const gpp_params&)

}  // namespace gpp
