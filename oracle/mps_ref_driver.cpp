// Runs the REFERENCE MPS reader (built from its sources by oracle/mps_ref.mk)
// on one file and writes what it parsed, for the parity tests of the
// engine's reader.  TEST INFRASTRUCTURE ONLY.
// usage: mps_ref_driver <model.mps> <out_dir>
// out_dir receives meta.txt (name, rows, cols, nnz, obj_constant) and raw
// little-endian arrays row_ptr (i64), col_idx (i32), csr_val, col_ptr (i64),
// row_idx (i32), csc_val, c, AL, AU, l, u (f64); on a parse error the driver
// prints the message and exits 1.
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "mps_reader/mpsreader.hpp"

template <class T>
static void save(const std::string& dir, const char* name, const std::vector<T>& v) {
  std::ofstream f(dir + "/" + name, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "usage: mps_ref_driver <model.mps> <out_dir>\n";
    return 2;
  }
  try {
    std::ifstream in(argv[1]);
    const auto model = mps_reader::read_mps(in);
    const auto& lp = model.lp;
    const std::string out = argv[2];
    std::ofstream meta(out + "/meta.txt");
    meta << std::setprecision(17) << "name " << model.name << "\nrows " << lp.num_rows() << "\ncols "
         << lp.num_cols() << "\nnnz " << lp.csr().values().size() << "\nobj_constant " << lp.obj_constant() << "\n";
    save(out, "row_ptr", lp.csr().row_ptr());
    save(out, "col_idx", lp.csr().col_idx());
    save(out, "csr_val", lp.csr().values());
    save(out, "col_ptr", lp.csc().col_ptr());
    save(out, "row_idx", lp.csc().row_idx());
    save(out, "csc_val", lp.csc().values());
    save(out, "c", lp.objective());
    save(out, "AL", lp.row_lower());
    save(out, "AU", lp.row_upper());
    save(out, "l", lp.col_lower());
    save(out, "u", lp.col_upper());
    return 0;
  } catch (const std::exception& e) {
    std::cout << "error " << e.what() << "\n";
    return 1;
  }
}
