// Turns gpp.h status codes back into the exceptions the reference's C++ API
// throws: std::runtime_error for CUDA and other runtime failures,
// std::length_error for offset overflow, std::invalid_argument for malformed
// input (cpp/include/gpu_preprocessor/offset.hpp:20-30,
// cpp/src/folding/folding.cu:79-81).
#pragma once

#include <stdexcept>
#include <string>

#include "gpp.h"

namespace gpu_preprocessor::detail {

inline void throw_on_status(int status, const char* what) {
  if (status == GPP_OK) return;
  std::string msg = std::string(what) + ": " + gpp_last_error();
  switch (status) {
    case GPP_ERR_LENGTH: throw std::length_error(msg);
    case GPP_ERR_INVALID: throw std::invalid_argument(msg);
    default: throw std::runtime_error(msg);
  }
}

}  // namespace gpu_preprocessor::detail
