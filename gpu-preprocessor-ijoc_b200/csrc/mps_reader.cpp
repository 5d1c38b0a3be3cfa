// Continuous-LP MPS reader (host code) and the upload of its model to a
// device gpp_lp.
//
// Restates the behaviour of GPU-Preprocessor's reader
// (cpp/mps_reader/src/io/mpsreader.cpp) so that the same file gives the same
// arrays, bit for bit:
//  - free format first, fixed-column format when free parsing fails
//    (:688-711); fixed fields at columns 2-3, 5-12, 15-22, 25-36, 40-47,
//    50-61 and the name from column 15 (:140-183);
//  - numbers by decimal digit accumulation with a library fallback
//    (:190-300), which is not correctly rounded and must not be replaced;
//  - the first N row is the objective, an RHS on it is the negated objective
//    constant, only the first RHS / RANGES / BOUNDS set counts (:343-517);
//  - RANGES and the bound types FR MI PL BV LO UP FX LI UI, and default bounds
//    [0, inf) ([0, 1] for columns inside INTORG markers), lower -inf when only
//    a negative upper bound is given (:452-538);
//  - a column's entries sorted by row (stable) and duplicates summed in file
//    order, zeros kept (:623-668); CSR by a stable transpose of that CSC;
//  - a lower bound above its upper bound rejects the model
//    (cpp/mps_reader/src/core/lp_model.cpp:21-56).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "mps_reader.hpp"

namespace gpp {

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

bool space(char c) { return std::isspace(static_cast<unsigned char>(c)) != 0; }

std::vector<std::string> tokens(const std::string& line) {
  std::vector<std::string> out;
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && space(line[i])) ++i;
    const size_t b = i;
    while (i < line.size() && !space(line[i])) ++i;
    if (b < i) out.push_back(line.substr(b, i - b));
  }
  return out;
}

std::string column_field(const std::string& line, size_t begin, size_t end) {
  if (line.size() <= begin) return {};
  std::string f = line.substr(begin, std::min(line.size(), end) - begin);
  const size_t a = f.find_first_not_of(" \t\r\n\v\f");
  if (a == std::string::npos) return {};
  const size_t z = f.find_last_not_of(" \t\r\n\v\f");
  return f.substr(a, z - a + 1);
}

// A line of the file: nothing (blank or comment), a section header, or data
// fields.
struct Line {
  enum Kind { kSkip, kHeader, kData } kind = kSkip;
  std::vector<std::string> fields;
};

Line read_line(const std::string& text, bool fixed) {
  Line l;
  const size_t first = text.find_first_not_of(" \t\r\n\v\f");
  if (first == std::string::npos || text[first] == '*' || text[first] == '&') return l;
  if (!space(text[0])) {
    l.kind = Line::kHeader;
    l.fields = tokens(text);
    if (l.fields.size() >= 2 && l.fields[0] == "OBJECT" && l.fields[1] == "BOUND") {
      l.fields = {"OBJECT BOUND"};
    } else if (fixed && !l.fields.empty() && l.fields[0] == "NAME") {
      const std::string name = column_field(text, 14, text.size());
      if (!name.empty()) l.fields = {"NAME", name};
    }
    return l;
  }
  l.kind = Line::kData;
  if (!fixed) {
    l.fields = tokens(text);
  } else {
    static const size_t cols[6][2] = {{1, 3}, {4, 12}, {14, 22}, {24, 36}, {39, 47}, {49, 61}};
    for (const auto& c : cols) {
      std::string f = column_field(text, c[0], c[1]);
      if (!f.empty()) l.fields.push_back(std::move(f));
    }
  }
  if (l.fields.empty()) l.kind = Line::kSkip;
  return l;
}

double library_number(const std::string& token) {
  std::string t = token;
  for (char& c : t)
    if (c == 'd' || c == 'D') c = 'E';
  size_t used = 0;
  const double v = std::stod(t, &used);
  if (used != t.size()) throw std::invalid_argument("invalid numeric token in MPS: " + token);
  return v;
}

// Sign, integer digits, fraction digits (each adding digit * 0.1^k, the
// scale kept by repeated multiplication), an optional e/E/d/D exponent applied
// by one multiplication or division by pow(10, e).  Anything else -- more
// than 18 digits, no digit, a malformed exponent, trailing characters -- goes
// to the library parser.
double mps_number(const std::string& s) {
  const size_t n = s.size();
  size_t i = 0;
  bool neg = false;
  if (i < n && (s[i] == '-' || s[i] == '+')) neg = s[i++] == '-';
  double v = 0.0, scale = 0.1;
  int digits = 0;
  auto digit = [](char c) { return c >= '0' && c <= '9'; };
  for (; i < n && digit(s[i]); ++i) {
    v = v * 10.0 + double(s[i] - '0');
    if (++digits > 18) return library_number(s);
  }
  if (i < n && s[i] == '.') {
    for (++i; i < n && digit(s[i]); ++i) {
      v += double(s[i] - '0') * scale;
      scale *= 0.1;
      if (++digits > 18) return library_number(s);
    }
  }
  if (digits == 0) return library_number(s);
  if (i < n) {
    if (s[i] != 'e' && s[i] != 'E' && s[i] != 'd' && s[i] != 'D') return library_number(s);
    ++i;
    bool eneg = false;
    if (i < n && (s[i] == '-' || s[i] == '+')) eneg = s[i++] == '-';
    int e = 0, edigits = 0;
    for (; i < n; ++i) {
      if (!digit(s[i])) return library_number(s);
      e = 10 * e + (s[i] - '0');
      ++edigits;
    }
    if (edigits == 0) return library_number(s);
    const double p = std::pow(10.0, e);
    v = eneg ? v / p : v * p;
  }
  return neg ? -v : v;
}

struct Row {
  char type;
  int index;   // -1 for N rows
};

struct Parser {
  std::string name, objective_row;
  std::unordered_map<std::string, Row> rows;
  std::unordered_map<std::string, int> cols;
  std::vector<char> row_type;
  std::vector<double> row_lo, row_hi;
  std::vector<std::vector<std::pair<int, double>>> entries;   // per column, file order
  std::vector<double> cost, col_lo, col_hi;                   // NaN: bound not given
  std::vector<char> marked_integer;
  double obj_constant = 0.0;
  std::string rhs_set, range_set, bound_set;

  const Row& row(const std::string& key, const char* where) const {
    const auto it = rows.find(key);
    if (it == rows.end()) throw std::invalid_argument(std::string("unknown MPS row in ") + where + ": " + key);
    return it->second;
  }

  int column(const std::string& key, bool integer) {
    const auto it = cols.find(key);
    if (it != cols.end()) return it->second;
    const int j = int(cols.size());
    cols.emplace(key, j);
    entries.emplace_back();
    cost.push_back(0.0);
    col_lo.push_back(std::numeric_limits<double>::quiet_NaN());
    col_hi.push_back(std::numeric_limits<double>::quiet_NaN());
    marked_integer.push_back(integer ? 1 : 0);
    return j;
  }

  void rows_line(const std::vector<std::string>& f) {
    if (f.size() < 2) throw std::invalid_argument("invalid ROWS entry");
    const char t = f[0].empty() ? '\0' : f[0][0];
    if (t == 'N') {
      if (objective_row.empty()) objective_row = f[1];
      rows.emplace(f[1], Row{'N', -1});
      return;
    }
    if (t != 'E' && t != 'G' && t != 'L') throw std::invalid_argument("unsupported MPS row type: " + std::string(1, t));
    rows.emplace(f[1], Row{t, int(row_type.size())});
    row_type.push_back(t);
    row_lo.push_back(t == 'L' ? -kInf : 0.0);
    row_hi.push_back(t == 'G' ? kInf : 0.0);
  }

  void columns_line(const std::vector<std::string>& f, bool integer) {
    if (f.size() < 3) throw std::invalid_argument("invalid COLUMNS entry");
    const int j = column(f[0], integer);
    for (size_t k = 1; k + 1 < f.size(); k += 2) {
      const double v = mps_number(f[k + 1]);
      const Row& r = row(f[k], "COLUMNS");
      if (r.index < 0) {
        if (f[k] == objective_row) cost[size_t(j)] += v;
        continue;
      }
      entries[size_t(j)].push_back({r.index, v});
    }
  }

  void rhs_line(const std::vector<std::string>& f) {
    if (f.size() < 3) throw std::invalid_argument("invalid RHS entry");
    if (rhs_set.empty()) rhs_set = f[0];
    if (f[0] != rhs_set) return;
    for (size_t k = 1; k + 1 < f.size(); k += 2) {
      const Row& r = row(f[k], "RHS");
      if (r.index < 0) {
        if (f[k] == objective_row) obj_constant = -mps_number(f[k + 1]);
        continue;
      }
      const double v = mps_number(f[k + 1]);
      const size_t i = size_t(r.index);
      if (r.type != 'L') row_lo[i] = v;
      if (r.type != 'G') row_hi[i] = v;
    }
  }

  void ranges_line(const std::vector<std::string>& f) {
    if (f.size() < 3) throw std::invalid_argument("invalid RANGES entry");
    if (range_set.empty()) range_set = f[0];
    if (f[0] != range_set) return;
    for (size_t k = 1; k + 1 < f.size(); k += 2) {
      const Row& r = row(f[k], "RANGES");
      const double v = mps_number(f[k + 1]);
      if (r.index < 0) continue;
      const size_t i = size_t(r.index);
      if (r.type == 'E') (v >= 0.0 ? row_hi[i] : row_lo[i]) += v;
      else if (r.type == 'L') row_lo[i] = row_hi[i] - std::fabs(v);
      else row_hi[i] = row_lo[i] + std::fabs(v);
    }
  }

  void bounds_line(const std::vector<std::string>& f) {
    if (f.size() < 3) throw std::invalid_argument("invalid BOUNDS entry");
    if (bound_set.empty()) bound_set = f[1];
    if (f[1] != bound_set) return;
    const auto it = cols.find(f[2]);
    if (it == cols.end()) throw std::invalid_argument("unknown MPS column in BOUNDS: " + f[2]);
    const size_t j = size_t(it->second);
    const std::string& t = f[0];
    if (t == "FR") { col_lo[j] = -kInf; col_hi[j] = kInf; return; }
    if (t == "MI") { col_lo[j] = -kInf; return; }
    if (t == "PL") { col_hi[j] = kInf; return; }
    if (t == "BV") { col_lo[j] = 0.0; col_hi[j] = 1.0; marked_integer[j] = 0; return; }
    if (f.size() < 4) throw std::invalid_argument("missing value for MPS bound type: " + t);
    const double v = mps_number(f[3]);
    if (t == "LO" || t == "LI") { col_lo[j] = v; if (t == "LI") marked_integer[j] = 0; }
    else if (t == "UP" || t == "UI") { col_hi[j] = v; if (t == "UI") marked_integer[j] = 0; }
    else if (t == "FX") { col_lo[j] = v; col_hi[j] = v; }
    else throw std::invalid_argument("unsupported MPS bound type: " + t);
  }

  void finish_bounds() {
    for (size_t j = 0; j < col_lo.size(); ++j) {
      const bool no_lo = std::isnan(col_lo[j]), no_hi = std::isnan(col_hi[j]);
      if (no_lo && no_hi) {
        col_lo[j] = 0.0;
        col_hi[j] = marked_integer[j] ? 1.0 : kInf;
      } else if (no_lo) {
        col_lo[j] = col_hi[j] < 0.0 ? -kInf : 0.0;
      } else if (no_hi) {
        col_hi[j] = kInf;
      }
    }
  }
};

enum class Section { kNone, kObjSense, kRows, kColumns, kRhs, kBounds, kRanges };

MpsModel parse(const std::vector<std::string>& lines, bool fixed) {
  Parser p;
  Section sec = Section::kNone;
  bool integer = false;
  for (const std::string& text : lines) {
    const Line l = read_line(text, fixed);
    if (l.kind == Line::kSkip) continue;
    const std::vector<std::string>& f = l.fields;
    if (l.kind == Line::kHeader) {
      const std::string& h = f[0];
      if (h == "NAME") { if (f.size() >= 2) p.name = f[1]; continue; }
      if (h == "ENDATA") break;
      if (h == "OBJSENSE") sec = Section::kObjSense;
      else if (h == "ROWS") sec = Section::kRows;
      else if (h == "COLUMNS") sec = Section::kColumns;
      else if (h == "RHS") sec = Section::kRhs;
      else if (h == "BOUNDS") sec = Section::kBounds;
      else if (h == "RANGES") sec = Section::kRanges;
      else if (h == "QUADOBJ" || h == "QMATRIX")
        throw std::invalid_argument("quadratic MPS sections are not supported by the MPS reader");
      else throw std::invalid_argument("unknown MPS section header: " + h);
      continue;
    }
    switch (sec) {
      case Section::kObjSense:
        if (f[0] == "MAX") throw std::invalid_argument("MPS OBJSENSE MAX is not supported by the MPS reader");
        break;
      case Section::kRows: p.rows_line(f); break;
      case Section::kColumns:
        if (f.size() >= 3 && f[1] == "'MARKER'") {
          if (f[2] == "'INTORG'") integer = true;
          else if (f[2] == "'INTEND'") integer = false;
          break;
        }
        p.columns_line(f, integer);
        break;
      case Section::kRhs: p.rhs_line(f); break;
      case Section::kBounds: p.bounds_line(f); break;
      case Section::kRanges: p.ranges_line(f); break;
      case Section::kNone: throw std::invalid_argument("MPS data entry outside a supported section");
    }
  }
  if (p.row_type.empty() && p.cols.empty()) throw std::invalid_argument("empty MPS model");
  p.finish_bounds();
  // A model with a lower bound above its upper bound is rejected, rows first
  // (the reference's LpModel constructor, lp_model.cpp:21-56).
  auto require = [](const char* lo_name, const char* hi_name, const std::vector<double>& lo,
                    const std::vector<double>& hi) {
    for (size_t k = 0; k < lo.size(); ++k)
      if (lo[k] > hi[k])
        throw std::invalid_argument(std::string(lo_name) + "[" + std::to_string(k) + "] exceeds " + hi_name + "[" +
                                    std::to_string(k) + "]");
  };
  require("row_lower", "row_upper", p.row_lo, p.row_hi);
  require("col_lower", "col_upper", p.col_lo, p.col_hi);

  MpsModel m;
  m.name = p.name;
  m.rows = int32_t(p.row_type.size());
  m.cols = int32_t(p.entries.size());
  m.col_ptr.assign(size_t(m.cols) + 1, 0);
  for (size_t j = 0; j < p.entries.size(); ++j) {
    auto& e = p.entries[j];
    std::stable_sort(e.begin(), e.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (size_t k = 0; k < e.size();) {
      double v = 0.0;
      size_t z = k;
      for (; z < e.size() && e[z].first == e[k].first; ++z) v += e[z].second;
      m.row_idx.push_back(e[k].first);
      m.csc_val.push_back(v);
      k = z;
    }
    m.col_ptr[j + 1] = int64_t(m.csc_val.size());
  }
  // CSR: rows in order, columns ascending within a row.
  const size_t nnz = m.csc_val.size();
  m.row_ptr.assign(size_t(m.rows) + 1, 0);
  for (int32_t i : m.row_idx) ++m.row_ptr[size_t(i) + 1];
  for (size_t i = 0; i < size_t(m.rows); ++i) m.row_ptr[i + 1] += m.row_ptr[i];
  m.col_idx.resize(nnz);
  m.csr_val.resize(nnz);
  std::vector<int64_t> next(m.row_ptr.begin(), m.row_ptr.end() - 1);
  for (int32_t j = 0; j < m.cols; ++j)
    for (int64_t q = m.col_ptr[size_t(j)]; q < m.col_ptr[size_t(j) + 1]; ++q) {
      const auto at = size_t(next[size_t(m.row_idx[size_t(q)])]++);
      m.col_idx[at] = j;
      m.csr_val[at] = m.csc_val[size_t(q)];
    }
  m.cost = std::move(p.cost);
  m.row_lower = std::move(p.row_lo);
  m.row_upper = std::move(p.row_hi);
  m.col_lower = std::move(p.col_lo);
  m.col_upper = std::move(p.col_hi);
  m.obj_constant = p.obj_constant;
  return m;
}

}  // namespace

MpsModel read_mps_text(const std::string& text) {
  std::vector<std::string> lines;
  std::istringstream in(text);
  for (std::string l; std::getline(in, l);) lines.push_back(std::move(l));
  try {
    return parse(lines, false);
  } catch (const std::exception& free_error) {
    const std::string why = free_error.what();
    try {
      return parse(lines, true);
    } catch (const std::exception&) {
      throw std::invalid_argument(why);
    }
  }
}

MpsModel read_mps_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::invalid_argument("cannot open MPS file: " + path);
  std::ostringstream all;
  all << f.rdbuf();
  return read_mps_text(all.str());
}

}  // namespace gpp
