// Host MPS model (see mps_reader.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace gpp {

struct MpsModel {
  std::string name;
  int32_t rows = 0, cols = 0;
  std::vector<int64_t> col_ptr;            // CSC
  std::vector<int32_t> row_idx;
  std::vector<double> csc_val;
  std::vector<int64_t> row_ptr;            // CSR
  std::vector<int32_t> col_idx;
  std::vector<double> csr_val;
  std::vector<double> cost, row_lower, row_upper, col_lower, col_upper;
  double obj_constant = 0.0;
};

MpsModel read_mps_text(const std::string& text);
MpsModel read_mps_file(const std::string& path);

}  // namespace gpp
