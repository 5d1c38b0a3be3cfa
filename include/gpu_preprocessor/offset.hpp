// Sparse offset type of the C++ layer over gpp.h.
//
// Mirrors cpp/include/gpu_preprocessor/offset.hpp:12-30 of GPU-Preprocessor:
// the global NnzOffset (int32 by default) and the checked conversions.  This
// engine is built with 32-bit offsets only (gpp_offset in gpp.h), so a
// consumer that asks for the 64-bit ABI is stopped at compile time instead of
// passing mismatched structs across the boundary.
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <stdexcept>

#include "gpp.h"

#ifndef GPUPREPROCESSOR_USE_INT64_NNZ
#define GPUPREPROCESSOR_USE_INT64_NNZ 0
#endif
#if GPUPREPROCESSOR_USE_INT64_NNZ
#error "this engine exports the 32-bit offset ABI only (gpp_offset is int32_t)"
#endif

using NnzOffset = gpp_offset;
static_assert(sizeof(NnzOffset) == 4, "gpp_offset must be int32_t");

inline NnzOffset checked_nnz_offset(std::int64_t count) {
  if (count < 0 || count > std::numeric_limits<NnzOffset>::max())
    throw std::length_error("nnz exceeds the 32-bit offset range of this build");
  return static_cast<NnzOffset>(count);
}

inline std::size_t checked_nnz_bytes(NnzOffset count, std::size_t element_size) {
  if (count < 0 || static_cast<std::uint64_t>(count) > std::numeric_limits<std::size_t>::max() / element_size)
    throw std::length_error("sparse allocation size overflow");
  return static_cast<std::size_t>(count) * element_size;
}
