// The model layer in front of the device solve, on the host: LpBuilder's
// standard form, the MPS reader and the exact presolve (include/prima_model.h).
// Compiled with -ffp-contract=off like the rest of the host code: the sums
// here are the reference's, in its order.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "prima_internal.h"
#include "prima_model.h"
#include "prima_nvtx.h"

namespace prima {
namespace model {

constexpr double kInf = std::numeric_limits<double>::infinity();

// Raised inside the model layer and turned into a return code at the C ABI.
struct Failure {
  int32_t code;
  std::string msg;
};

[[noreturn]] void require_fail(const std::string &m) {
  throw Failure{PRIMA_ERR_INVALID_ARGUMENT, "requirement failed: " + m};
}
[[noreturn]] void parse_fail(const std::string &m) { throw Failure{PRIMA_ERR_PARSE, m}; }

std::string num(double v) {
  if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
  char b[64];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}

using Terms = std::vector<std::pair<int32_t, double>>;

// A standard-form LpProblem that owns its arrays.
struct Lp {
  int32_t n = 0, m = 0, neq = 0;
  std::vector<int32_t> rp{0}, ci;
  std::vector<double> v, c, q, lo, hi;
  double offset = 0.0;

  prima_lp view() const {
    prima_lp lp;
    lp.num_variables = n;
    lp.num_constraints = m;
    lp.num_equalities = neq;
    lp.pad = 0;
    lp.row_ptr = rp.data();
    lp.col_idx = ci.data();
    lp.values = v.data();
    lp.objective = c.data();
    lp.rhs = q.data();
    lp.lower = lo.data();
    lp.upper = hi.data();
    lp.objective_offset = offset;
    return lp;
  }
};

// SparseMatrix.fromTriplets (SparseMatrix.scala:204-260): non-finite entries
// rejected, a stable sort by (row, column), duplicates summed in order of
// appearance, exact zeros dropped.
struct Triplet {
  int32_t r, c;
  double v;
};

void from_triplets(int32_t rows, int32_t cols, std::vector<Triplet> &t, Lp *out) {
  for (const Triplet &e : t)
    if (!std::isfinite(e.v))
      require_fail("entry at (" + std::to_string(e.r) + ", " + std::to_string(e.c) + ") is not finite");
  std::vector<int64_t> start((size_t)rows + 1, 0);
  for (const Triplet &e : t) start[(size_t)e.r + 1]++;
  for (int32_t r = 0; r < rows; r++) start[(size_t)r + 1] += start[(size_t)r];
  std::vector<Triplet> by_row(t.size());
  {
    std::vector<int64_t> at(start.begin(), start.end() - 1);
    for (const Triplet &e : t) by_row[(size_t)at[(size_t)e.r]++] = e;  // stable within a row
  }
  out->rp.assign((size_t)rows + 1, 0);
  out->ci.clear();
  out->v.clear();
  out->ci.reserve(t.size());
  out->v.reserve(t.size());
  for (int32_t r = 0; r < rows; r++) {
    auto b = by_row.begin() + start[(size_t)r], e = by_row.begin() + start[(size_t)r + 1];
    std::stable_sort(b, e, [](const Triplet &x, const Triplet &y) { return x.c < y.c; });
    for (auto k = b; k != e;) {
      double acc = k->v;
      auto g = k + 1;
      for (; g != e && g->c == k->c; ++g) acc = acc + g->v;
      if (acc != 0.0) {
        out->ci.push_back(k->c);
        out->v.push_back(acc);
      }
      k = g;
    }
    if (out->ci.size() > (size_t)std::numeric_limits<int32_t>::max()) require_fail("more than 2^31 - 1 nonzeros");
    out->rp[(size_t)r + 1] = (int32_t)out->ci.size();
  }
  out->m = rows;
  out->n = cols;
}

// LpBuilder (LpProblem.scala:152-248): rows as lo <= a'x <= hi; build() puts
// equalities first in insertion order, then the rest, `<=` rows negated and
// ranges split into a'x >= lo and -a'x >= -hi.
class Builder {
 public:
  explicit Builder(int32_t n) : n_(n), c_((size_t)n, 0.0), lo_((size_t)n, -kInf), hi_((size_t)n, kInf) {}

  void objective(int32_t j, double v) {
    check(j);
    c_[(size_t)j] = v;
  }
  void offset(double v) { offset_ = v; }
  void bounds(int32_t j, double lo, double hi) {
    check(j);
    if (!(lo <= hi))
      require_fail("variable " + std::to_string(j) + " has empty bound interval [" + num(lo) + ", " + num(hi) + "]");
    lo_[(size_t)j] = lo;
    hi_[(size_t)j] = hi;
  }
  void constraint(Terms terms, double lo, double hi) {
    if (!(lo <= hi)) require_fail("constraint has empty range [" + num(lo) + ", " + num(hi) + "]");
    if (lo == -kInf && hi == kInf) require_fail("constraint is unbounded on both sides and would have no effect");
    for (const auto &t : terms) check(t.first);
    rows_.push_back(Row{std::move(terms), lo, hi});
  }

  // kinds/first/second: the RowTranslation, one entry per constraint() call.
  void build(Lp *out, std::vector<int32_t> *kind = nullptr, std::vector<int32_t> *first = nullptr,
             std::vector<int32_t> *second = nullptr) {
    std::vector<Triplet> t;
    std::vector<double> rhs;
    size_t total = 0;
    for (const Row &r : rows_) total += r.terms.size();
    t.reserve(total + total / 8);
    auto emit = [&](const Terms &co, double sign, double value) {
      const int32_t r = (int32_t)rhs.size();
      for (const auto &e : co) t.push_back(Triplet{r, e.first, sign * e.second});
      rhs.push_back(sign * value);
      return r;
    };
    const size_t k = rows_.size();
    if (kind) {
      kind->assign(k, 0);
      first->assign(k, -1);
      second->assign(k, -1);
    }
    for (size_t i = 0; i < k; i++) {
      const Row &r = rows_[i];
      if (r.lo == r.hi) {
        const int32_t a = emit(r.terms, 1.0, r.lo);
        if (kind) (*kind)[i] = 0, (*first)[i] = a;
      }
    }
    const int32_t neq = (int32_t)rhs.size();
    for (size_t i = 0; i < k; i++) {
      const Row &r = rows_[i];
      if (r.lo == r.hi) continue;
      const bool has_lo = r.lo != -kInf, has_hi = r.hi != kInf;
      if (has_lo && has_hi) {
        const int32_t a = emit(r.terms, 1.0, r.lo);
        const int32_t b = emit(r.terms, -1.0, r.hi);
        if (kind) (*kind)[i] = 2, (*first)[i] = a, (*second)[i] = b;
      } else if (has_lo) {
        const int32_t a = emit(r.terms, 1.0, r.lo);
        if (kind) (*kind)[i] = 0, (*first)[i] = a;
      } else {
        const int32_t a = emit(r.terms, -1.0, r.hi);
        if (kind) (*kind)[i] = 1, (*first)[i] = a;
      }
    }
    if (rhs.size() > (size_t)std::numeric_limits<int32_t>::max()) require_fail("more than 2^31 - 1 rows");
    from_triplets((int32_t)rhs.size(), n_, t, out);
    out->neq = neq;
    out->q = std::move(rhs);
    out->c = c_;
    out->lo = lo_;
    out->hi = hi_;
    out->offset = offset_;
  }

 private:
  struct Row {
    Terms terms;
    double lo, hi;
  };
  void check(int32_t j) const {
    if (!(j >= 0 && j < n_))
      require_fail("variable index " + std::to_string(j) + " out of range [0, " + std::to_string(n_) + ")");
  }
  int32_t n_;
  std::vector<double> c_, lo_, hi_;
  double offset_ = 0.0;
  std::vector<Row> rows_;
};

// ---- MPS --------------------------------------------------------------------

// Java's trim: every character at or below U+0020 goes from both ends.
std::string java_trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && (unsigned char)s[a] <= 0x20) a++;
  while (b > a && (unsigned char)s[b - 1] <= 0x20) b--;
  return s.substr(a, b - a);
}

// split("\\s+") on a trimmed line: \s is [ \t\n\x0B\f\r].
bool java_space(char ch) {
  return ch == ' ' || ch == '\t' || ch == '\n' || ch == '\x0b' || ch == '\f' || ch == '\r';
}

std::vector<std::string> tokens_of(const std::string &trimmed) {
  std::vector<std::string> out;
  size_t i = 0;
  const size_t n = trimmed.size();
  while (i < n) {
    size_t j = i;
    while (j < n && !java_space(trimmed[j])) j++;
    out.push_back(trimmed.substr(i, j - i));
    while (j < n && java_space(trimmed[j])) j++;
    i = j;
  }
  if (out.empty()) out.push_back(std::string());
  return out;
}

std::string upper(std::string s) {
  for (char &ch : s) ch = (char)std::toupper((unsigned char)ch);
  return s;
}

// String.toDoubleOption (java.lang.Double.parseDouble's grammar): an optional
// sign, then NaN, Infinity, a decimal with optional exponent, or a hex float
// with a binary exponent; an optional f/F/d/D suffix.  Conversion by strtod,
// which rounds correctly like the JVM.
bool parse_double(const std::string &tok, double *out) {
  const std::string s = java_trim(tok);
  size_t i = 0;
  const size_t n = s.size();
  bool neg = false;
  if (i < n && (s[i] == '+' || s[i] == '-')) neg = s[i++] == '-';
  const std::string rest = s.substr(i);
  if (rest == "NaN") {
    *out = std::numeric_limits<double>::quiet_NaN();
    return true;
  }
  if (rest == "Infinity") {
    *out = neg ? -kInf : kInf;
    return true;
  }
  size_t end = n;
  if (end > i && (s[end - 1] == 'f' || s[end - 1] == 'F' || s[end - 1] == 'd' || s[end - 1] == 'D')) end--;
  auto digits = [&](size_t &k, bool hex) {
    const size_t k0 = k;
    while (k < end && (hex ? std::isxdigit((unsigned char)s[k]) : std::isdigit((unsigned char)s[k]))) k++;
    return k - k0;
  };
  size_t k = i;
  bool ok = false;
  if (k + 1 < end && s[k] == '0' && (s[k + 1] == 'x' || s[k + 1] == 'X')) {
    // hex: 0x h* [. h*] p [+-] d+, at least one hex digit
    k += 2;
    size_t nd = digits(k, true);
    if (k < end && s[k] == '.') {
      k++;
      nd += digits(k, true);
    }
    if (nd > 0 && k < end && (s[k] == 'p' || s[k] == 'P')) {
      k++;
      if (k < end && (s[k] == '+' || s[k] == '-')) k++;
      ok = digits(k, false) > 0 && k == end;
    }
  } else {
    size_t nd = digits(k, false);
    if (k < end && s[k] == '.') {
      k++;
      nd += digits(k, false);
    }
    if (nd > 0) {
      if (k < end && (s[k] == 'e' || s[k] == 'E')) {
        k++;
        if (k < end && (s[k] == '+' || s[k] == '-')) k++;
        ok = digits(k, false) > 0 && k == end;
      } else {
        ok = k == end;
      }
    }
  }
  if (!ok) return false;
  const std::string body = s.substr(0, end);
  char *stop = nullptr;
  *out = std::strtod(body.c_str(), &stop);
  return stop == body.c_str() + body.size();
}

struct MpsRow {
  std::string name;
  char sense = 'E';
  double rhs = 0.0;
  bool has_range = false;
  double range = 0.0;
  Terms entries;
};

struct MpsCol {
  std::string name;
  int32_t index = 0;
  double lower = 0.0, upper = kInf, objective = 0.0;
  bool integer = false, lower_explicit = false;
};

struct Instance {
  std::string name;
  Lp lp;
  std::vector<int32_t> kind, first, second;
  std::vector<std::string> row_names, col_names;
  std::vector<int32_t> integer_cols;
};

// MpsReader.fromLines (MpsReader.scala:91-235).
class MpsReader {
 public:
  explicit MpsReader(std::string fallback) : name_(std::move(fallback)) {}

  void line(const std::string &raw) {
    std::string line = raw;
    std::replace(line.begin(), line.end(), '\t', ' ');
    const std::string trimmed = java_trim(line);
    if (trimmed.empty() || line[0] == '*') return;
    const std::vector<std::string> tok = tokens_of(trimmed);
    if (line[0] != ' ') {
      section_ = upper(tok[0]);
      if (section_ == "NAME" && tok.size() > 1) name_ = tok[1];
      else if (section_ == "OBJSENSE" && tok.size() > 1) check_objsense(tok[1]);
      return;
    }
    if (section_ == "ROWS") rows_line(tok, line);
    else if (section_ == "COLUMNS") columns_line(tok, line);
    else if (section_ == "RHS" || section_ == "RANGES") rhs_line(tok, line);
    else if (section_ == "BOUNDS") bounds_line(tok, line);
    else if (section_ == "OBJSENSE") check_objsense(tok[0]);
    else if (section_ == "ENDATA" || section_.empty()) {
    } else {
      parse_fail("unexpected data in section '" + section_ + "'");
    }
  }

  Instance finish() {
    if (objective_.empty()) parse_fail("no objective row (an N row) was declared");
    Instance out;
    out.name = name_;
    Builder b((int32_t)cols_.size());
    b.offset(obj_constant_);
    for (const MpsCol &c : cols_) {
      b.objective(c.index, c.objective);
      if (c.lower > c.upper)
        parse_fail("column '" + c.name + "' has empty bounds [" + num(c.lower) + ", " + num(c.upper) + "]");
      b.bounds(c.index, c.lower, c.upper);
    }
    for (const MpsRow &r : rows_) {
      double lo, hi;
      bracket(r, &lo, &hi);
      b.constraint(r.entries, lo, hi);
      out.row_names.push_back(r.name);
    }
    b.build(&out.lp, &out.kind, &out.first, &out.second);
    for (const MpsCol &c : cols_) {
      out.col_names.push_back(c.name);
      if (c.integer) out.integer_cols.push_back(c.index);
    }
    return out;
  }

 private:
  static void check_objsense(const std::string &tok) {
    if (upper(tok).rfind("MAX", 0) == 0) parse_fail("OBJSENSE MAX is not supported; the solver minimises");
  }

  static double number(const std::string &tok, const std::string &line) {
    double v;
    if (!parse_double(tok, &v)) parse_fail("'" + tok + "' is not a number, in: '" + line + "'");
    return v;
  }

  static std::vector<std::pair<std::string, double>> pairs(const std::vector<std::string> &f, size_t from,
                                                           const std::string &line, const std::string &section) {
    if ((f.size() - from) % 2) parse_fail(section + " entry has an unpaired field: '" + line + "'");
    std::vector<std::pair<std::string, double>> out;
    for (size_t i = from; i < f.size(); i += 2) out.emplace_back(f[i], number(f[i + 1], line));
    return out;
  }

  MpsCol &column(const std::string &name) {
    auto it = col_index_.find(name);
    if (it != col_index_.end()) return cols_[it->second];
    col_index_.emplace(name, cols_.size());
    MpsCol col;
    col.name = name;
    col.index = (int32_t)cols_.size();
    cols_.push_back(col);
    return cols_.back();
  }

  MpsRow *row(const std::string &name, const char *context) {
    if (free_.count(name) || name == objective_) return nullptr;
    auto it = row_index_.find(name);
    if (it == row_index_.end()) parse_fail(std::string(context) + " refers to unknown row '" + name + "'");
    return &rows_[it->second];
  }

  void rows_line(const std::vector<std::string> &tok, const std::string &line) {
    if (tok.size() < 2) parse_fail("malformed ROWS entry: '" + line + "'");
    const std::string kind = upper(tok[0]), &name = tok[1];
    if (kind == "N") {
      if (objective_.empty()) objective_ = name;
      else free_.insert(name);
    } else if (kind == "L" || kind == "G" || kind == "E") {
      MpsRow r;
      r.name = name;
      r.sense = kind[0];
      auto it = row_index_.find(name);
      if (it != row_index_.end()) {
        rows_[it->second] = r;  // redeclared: a fresh row in the old place
      } else {
        row_index_.emplace(name, rows_.size());
        rows_.push_back(r);
      }
    } else {
      parse_fail("unknown row type '" + kind + "' for row '" + name + "'");
    }
  }

  void columns_line(const std::vector<std::string> &tok, const std::string &line) {
    if (std::find(tok.begin(), tok.end(), "'MARKER'") != tok.end()) {
      bool start = false, stop = false;
      for (const std::string &t : tok) {
        const std::string u = upper(t);
        start = start || u == "'INTORG'";
        stop = stop || u == "'INTEND'";
      }
      if (start) integer_block_ = true;
      else if (stop) integer_block_ = false;
      return;
    }
    if (tok.size() < 3) parse_fail("malformed COLUMNS entry: '" + line + "'");
    const auto entries = pairs(tok, 1, line, "COLUMNS");
    MpsCol &col = column(tok[0]);
    if (integer_block_) col.integer = true;
    const int32_t index = col.index;
    for (const auto &e : entries) {
      if (e.first == objective_) {
        cols_[(size_t)index].objective += e.second;
      } else if (!free_.count(e.first)) {
        MpsRow *r = row(e.first, "COLUMNS");
        if (r) r->entries.emplace_back(index, e.second);
      }
    }
  }

  void rhs_line(const std::vector<std::string> &tok, const std::string &line) {
    const size_t from = tok.size() % 2 == 1 ? 1 : 0;
    const bool rhs = section_ == "RHS";
    for (const auto &e : pairs(tok, from, line, section_)) {
      if (rhs) {
        if (e.first == objective_) {
          obj_constant_ = -e.second;
        } else if (!free_.count(e.first)) {
          MpsRow *r = row(e.first, "RHS");
          if (r) r->rhs = e.second;
        }
      } else {
        MpsRow *r = row(e.first, "RANGES");
        if (r) r->has_range = true, r->range = e.second;
      }
    }
  }

  void bounds_line(const std::vector<std::string> &tok, const std::string &line) {
    if (tok.size() < 2) parse_fail("malformed BOUNDS entry: '" + line + "'");
    const std::string kind = upper(tok[0]);
    const bool valueless = kind == "FR" || kind == "MI" || kind == "PL" || kind == "BV";
    const size_t stop = valueless ? tok.size() : std::max<size_t>(2, tok.size() - 1);
    const std::string *name = nullptr;
    std::string tried;
    for (size_t i = 1; i < stop && i < tok.size(); i++) {
      tried += (i > 1 ? ", " : "") + tok[i];
      if (!name && col_index_.count(tok[i])) name = &tok[i];
    }
    if (!name) parse_fail("BOUNDS names no column declared in COLUMNS (tried " + tried + ") in: '" + line + "'");
    if (tok.size() > 4) parse_fail("BOUNDS entry carries more fields than one bound uses: '" + line + "'");
    MpsCol &col = cols_[col_index_[*name]];
    if (kind == "UP") {
      const double v = number(tok.back(), line);
      col.upper = v;
      if (v < 0.0 && !col.lower_explicit) col.lower = -kInf;
    } else if (kind == "LO") {
      col.lower = number(tok.back(), line);
      col.lower_explicit = true;
    } else if (kind == "FX") {
      const double v = number(tok.back(), line);
      col.lower = col.upper = v;
      col.lower_explicit = true;
    } else if (kind == "FR") {
      col.lower = -kInf, col.upper = kInf, col.lower_explicit = true;
    } else if (kind == "MI") {
      col.lower = -kInf, col.lower_explicit = true;
    } else if (kind == "PL") {
      col.upper = kInf;
    } else if (kind == "BV") {
      col.lower = 0.0, col.upper = 1.0, col.integer = true, col.lower_explicit = true;
    } else if (kind == "LI") {
      col.lower = number(tok.back(), line), col.integer = true, col.lower_explicit = true;
    } else if (kind == "UI") {
      col.upper = number(tok.back(), line), col.integer = true;
    } else {
      parse_fail("unknown bound type '" + kind + "' on '" + *name + "'");
    }
  }

  // Row sense, right-hand side and optional range as two-sided bounds
  // (MpsReader.scala:300-316).
  static void bracket(const MpsRow &r, double *lo, double *hi) {
    if (!r.has_range) {
      *lo = r.sense == 'L' ? -kInf : r.rhs;
      *hi = r.sense == 'G' ? kInf : r.rhs;
      return;
    }
    const double w = std::fabs(r.range);
    if (r.sense == 'G') *lo = r.rhs, *hi = r.rhs + w;
    else if (r.sense == 'L') *lo = r.rhs - w, *hi = r.rhs;
    else if (r.range >= 0.0) *lo = r.rhs, *hi = r.rhs + w;
    else *lo = r.rhs - w, *hi = r.rhs;
  }

  std::string name_, objective_, section_;
  double obj_constant_ = 0.0;
  bool integer_block_ = false;
  std::vector<MpsRow> rows_;
  std::unordered_map<std::string, size_t> row_index_;
  std::vector<MpsCol> cols_;
  std::unordered_map<std::string, size_t> col_index_;
  std::unordered_set<std::string> free_;
};

// Lines end at LF, CR or CR LF, as Source.getLines and linesIterator split them.
Instance read_text(const char *text, int64_t length, const std::string &fallback) {
  NvtxRange range("prima: read MPS");
  MpsReader reader(fallback);
  int64_t i = 0;
  while (i < length) {
    int64_t j = i;
    while (j < length && text[j] != '\n' && text[j] != '\r') j++;
    reader.line(std::string(text + i, (size_t)(j - i)));
    if (j < length && text[j] == '\r' && j + 1 < length && text[j + 1] == '\n') j++;
    i = j + 1;
  }
  return reader.finish();
}

// ---- presolve (Presolve.scala:199-408) --------------------------------------

struct Undo {
  enum Kind { kFixed, kEmptyCol, kEmptyRow, kSingleton } kind;
  int32_t r, j;
  double value, coef, bound;  // fixed/empty: value (and cost in coef); singleton: coefficient, bound
};

struct Presolved {
  Lp original;
  std::vector<int32_t> tp, tci;  // the original's transpose (rows ascending per column)
  std::vector<double> tv;
  int32_t fixed = 0, empty_cols = 0, empty_rows = 0, singletons = 0, passes = 0;
  bool infeasible = false, unbounded_if_feasible = false;
  std::vector<Undo> undo;  // oldest first
  std::vector<int32_t> column_map, row_map;
  Lp reduced;
};

void transpose(const Lp &a, std::vector<int32_t> *tp, std::vector<int32_t> *tci, std::vector<double> *tv) {
  tp->assign((size_t)a.n + 1, 0);
  for (int32_t k = 0; k < a.rp[(size_t)a.m]; k++) (*tp)[(size_t)a.ci[(size_t)k] + 1]++;
  for (int32_t j = 0; j < a.n; j++) (*tp)[(size_t)j + 1] += (*tp)[(size_t)j];
  tci->resize(a.ci.size());
  tv->resize(a.v.size());
  std::vector<int32_t> at(tp->begin(), tp->end() - 1);
  for (int32_t r = 0; r < a.m; r++)
    for (int32_t k = a.rp[(size_t)r]; k < a.rp[(size_t)r + 1]; k++) {
      const int32_t p = at[(size_t)a.ci[(size_t)k]]++;
      (*tci)[(size_t)p] = r;
      (*tv)[(size_t)p] = a.v[(size_t)k];
    }
}

void presolve(Presolved &P, int32_t max_passes) {
  NvtxRange range("prima: presolve");
  const Lp &A = P.original;
  const int32_t n = A.n, m = A.m, neq = A.neq;
  transpose(A, &P.tp, &P.tci, &P.tv);
  std::vector<char> col_alive((size_t)n, 1), row_alive((size_t)m, 1);
  std::vector<double> lower = A.lo, upper = A.hi, fixed_shift((size_t)m, 0.0), fixed_value((size_t)n, 0.0);

  auto fix_column = [&](int32_t j, double value) {
    col_alive[(size_t)j] = 0;
    fixed_value[(size_t)j] = value;
    P.fixed++;
    P.undo.push_back(Undo{Undo::kFixed, -1, j, value, 0.0, 0.0});
    for (int32_t k = P.tp[(size_t)j]; k < P.tp[(size_t)j + 1]; k++) {
      const int32_t r = P.tci[(size_t)k];
      if (row_alive[(size_t)r]) fixed_shift[(size_t)r] += P.tv[(size_t)k] * value;
    }
  };
  auto col_has_live_row = [&](int32_t j) {
    for (int32_t k = P.tp[(size_t)j]; k < P.tp[(size_t)j + 1]; k++)
      if (row_alive[(size_t)P.tci[(size_t)k]]) return true;
    return false;
  };

  bool changed = true;
  while (changed && P.passes < max_passes && !P.infeasible) {
    changed = false;
    P.passes++;
    for (int32_t j = 0; j < n; j++)  // a column whose bounds coincide (:237-242)
      if (col_alive[(size_t)j] && lower[(size_t)j] == upper[(size_t)j] && std::isfinite(lower[(size_t)j])) {
        fix_column(j, lower[(size_t)j]);
        changed = true;
      }
    for (int32_t r = 0; r < m && !P.infeasible; r++) {
      if (!row_alive[(size_t)r]) continue;
      int32_t live = 0, jj = -1;
      double aa = 0.0;
      for (int32_t k = A.rp[(size_t)r]; k < A.rp[(size_t)r + 1] && live < 2; k++)
        if (col_alive[(size_t)A.ci[(size_t)k]]) {
          if (live == 0) jj = A.ci[(size_t)k], aa = A.v[(size_t)k];
          live++;
        }
      const double adjusted = A.q[(size_t)r] - fixed_shift[(size_t)r];
      const bool is_eq = r < neq;
      if (live == 0) {  // an empty row holds or proves infeasibility (:252-267)
        const double magnitude = std::max(std::fabs(A.q[(size_t)r]), std::fabs(fixed_shift[(size_t)r]));
        const double scale = std::isfinite(magnitude) ? 1e-9 * std::max(1.0, magnitude) : 1e-9;
        const bool holds = is_eq ? std::fabs(adjusted) <= scale : adjusted <= scale;
        if (!holds) {
          P.infeasible = true;
        } else {
          row_alive[(size_t)r] = 0;
          P.empty_rows++;
          P.undo.push_back(Undo{Undo::kEmptyRow, r, -1, 0.0, 0.0, 0.0});
          changed = true;
        }
      } else if (live == 1) {  // a bound in disguise (:268-292)
        const double bound = adjusted / aa;
        double lo = lower[(size_t)jj], hi = upper[(size_t)jj];
        if (is_eq) {
          lo = std::max(lo, bound);
          hi = std::min(hi, bound);
        } else if (aa > 0.0) {
          lo = std::max(lo, bound);
        } else {
          hi = std::min(hi, bound);
        }
        bool contradictory;
        if (!std::isfinite(lo) || !std::isfinite(hi)) contradictory = lo > hi;
        else contradictory = lo > hi + 1e-9 * std::max(1.0, std::max(std::fabs(lo), std::fabs(hi)));
        if (contradictory) {
          P.infeasible = true;
        } else {
          lower[(size_t)jj] = lo;
          upper[(size_t)jj] = std::max(hi, lo);
          row_alive[(size_t)r] = 0;
          P.singletons++;
          P.undo.push_back(Undo{Undo::kSingleton, r, jj, 0.0, aa, bound});
          changed = true;
        }
      }
    }
    if (P.infeasible) break;
    for (int32_t j = 0; j < n; j++) {  // a column in no live row (:294-323)
      if (!col_alive[(size_t)j] || col_has_live_row(j)) continue;
      const double cost = A.c[(size_t)j];
      double at;
      if (cost > 0.0) at = lower[(size_t)j];
      else if (cost < 0.0) at = upper[(size_t)j];
      else if (std::isfinite(lower[(size_t)j])) at = lower[(size_t)j];
      else if (std::isfinite(upper[(size_t)j])) at = upper[(size_t)j];
      else at = 0.0;
      col_alive[(size_t)j] = 0;
      P.empty_cols++;
      if (!std::isfinite(at)) {
        P.unbounded_if_feasible = true;
        P.undo.push_back(Undo{Undo::kEmptyCol, -1, j, 0.0, cost, 0.0});
      } else {
        fixed_value[(size_t)j] = at;
        P.undo.push_back(Undo{Undo::kEmptyCol, -1, j, at, cost, 0.0});
      }
      changed = true;
    }
  }
  if (P.infeasible) return;

  std::vector<int32_t> new_col((size_t)n, -1);
  for (int32_t j = 0; j < n; j++)
    if (col_alive[(size_t)j]) new_col[(size_t)j] = (int32_t)P.column_map.size(), P.column_map.push_back(j);
  for (int32_t r = 0; r < m; r++)
    if (row_alive[(size_t)r]) P.row_map.push_back(r);
  Builder b((int32_t)P.column_map.size());
  double offset = A.offset;
  for (int32_t j = 0; j < n; j++)
    if (!col_alive[(size_t)j]) offset += A.c[(size_t)j] * fixed_value[(size_t)j];
  b.offset(offset);
  for (size_t i = 0; i < P.column_map.size(); i++) {
    const int32_t old = P.column_map[i];
    b.objective((int32_t)i, A.c[(size_t)old]);
    b.bounds((int32_t)i, lower[(size_t)old], upper[(size_t)old]);
  }
  for (int32_t old : P.row_map) {
    Terms entries;
    for (int32_t k = A.rp[(size_t)old]; k < A.rp[(size_t)old + 1]; k++) {
      const int32_t j = A.ci[(size_t)k];
      if (col_alive[(size_t)j]) entries.emplace_back(new_col[(size_t)j], A.v[(size_t)k]);
    }
    const double value = A.q[(size_t)old] - fixed_shift[(size_t)old];
    if (old < neq) b.constraint(std::move(entries), value, value);
    else b.constraint(std::move(entries), value, kInf);
  }
  b.build(&P.reduced);
}

// PresolveResult.restore (Presolve.scala:108-191), the vectors.
void restore(const Presolved &P, const double *x, const double *y, const double *rc, double *xo, double *yo,
             double *rco) {
  const Lp &A = P.original;
  const double nan = std::numeric_limits<double>::quiet_NaN();
  std::fill(xo, xo + A.n, 0.0);
  std::fill(rco, rco + A.n, 0.0);
  std::fill(yo, yo + A.m, 0.0);
  for (size_t i = 0; i < P.column_map.size(); i++) {
    xo[P.column_map[i]] = x[i];
    rco[P.column_map[i]] = rc[i];
  }
  for (size_t i = 0; i < P.row_map.size(); i++) yo[P.row_map[i]] = y[i];
  for (auto u = P.undo.rbegin(); u != P.undo.rend(); ++u) {  // newest first
    switch (u->kind) {
      case Undo::kFixed:
        xo[u->j] = u->value;
        rco[u->j] = nan;  // recomputed from the restored duals below
        break;
      case Undo::kEmptyCol:
        xo[u->j] = u->value;
        rco[u->j] = u->coef;
        break;
      case Undo::kEmptyRow:
        yo[u->r] = 0.0;
        break;
      case Undo::kSingleton: {
        const double bound = u->bound, a = u->coef;
        const bool on_bound = std::fabs(xo[u->j] - bound) <= 1e-7 * std::max(1.0, std::fabs(bound));
        if (on_bound && a != 0.0 && !std::isnan(rco[u->j]) && rco[u->j] != 0.0) {
          const double price = rco[u->j] / a;
          yo[u->r] = price;
          rco[u->j] = rco[u->j] - a * price;
        } else {
          yo[u->r] = 0.0;
        }
        break;
      }
    }
  }
  for (int32_t j = 0; j < A.n; j++) {  // K'y in row order, for the columns still unpriced
    if (!std::isnan(rco[j])) continue;
    double s = 0.0;
    for (int32_t k = P.tp[(size_t)j]; k < P.tp[(size_t)j + 1]; k++) s = s + P.tv[(size_t)k] * yo[P.tci[(size_t)k]];
    rco[j] = A.c[(size_t)j] - s;
  }
}

Lp copy_lp(const prima_lp *lp) {
  if (!lp) require_fail("lp is NULL");
  if (lp->num_variables < 0 || lp->num_constraints < 0 || lp->num_equalities < 0 ||
      lp->num_equalities > lp->num_constraints)
    require_fail("inconsistent problem dimensions");
  Lp out;
  out.n = lp->num_variables;
  out.m = lp->num_constraints;
  out.neq = lp->num_equalities;
  const size_t n = (size_t)out.n, m = (size_t)out.m;
  if (m && !lp->row_ptr) require_fail("row_ptr is NULL");
  out.rp.assign(lp->row_ptr, lp->row_ptr + m + 1);
  if (out.rp[0] != 0) require_fail("row_ptr[0] must be 0");
  for (size_t r = 0; r < m; r++)
    if (out.rp[r + 1] < out.rp[r]) require_fail("row_ptr must be non-decreasing");
  const size_t nnz = (size_t)out.rp[m];
  out.ci.assign(lp->col_idx, lp->col_idx + nnz);
  out.v.assign(lp->values, lp->values + nnz);
  for (int32_t j : out.ci)
    if (j < 0 || j >= out.n) require_fail("column index " + std::to_string(j) + " out of range");
  out.c.assign(lp->objective, lp->objective + n);
  out.q.assign(lp->rhs, lp->rhs + m);
  out.lo.assign(lp->lower, lp->lower + n);
  out.hi.assign(lp->upper, lp->upper + n);
  out.offset = lp->objective_offset;
  return out;
}

template <typename F>
int32_t guarded(F &&f) {
  try {
    f();
    clear_error();
    return PRIMA_OK;
  } catch (const Failure &e) {
    set_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc &) {
    set_error("out of host memory");
    return PRIMA_ERR_OUT_OF_MEMORY;
  }
}

}  // namespace model
}  // namespace prima

struct prima_mps_instance {
  prima::model::Instance inst;
};

struct prima_presolved {
  prima::model::Presolved p;
};

using prima::model::Failure;
using prima::model::guarded;
using prima::model::require_fail;

extern "C" int32_t prima_mps_read(const char *text, int64_t length, const char *fallback_name,
                                  prima_mps_instance **out) {
  return guarded([&] {
    if (!out) require_fail("out is NULL");
    *out = nullptr;
    if (!text && length) require_fail("text is NULL");
    if (length < 0) require_fail("length must be non-negative");
    auto h = std::make_unique<prima_mps_instance>();
    h->inst = prima::model::read_text(text, length, fallback_name ? fallback_name : "inline");
    *out = h.release();
  });
}

extern "C" int32_t prima_mps_read_file(const char *path, prima_mps_instance **out) {
  return guarded([&] {
    if (!out || !path) require_fail("path or out is NULL");
    *out = nullptr;
    std::ifstream f(path, std::ios::binary);
    if (!f) throw Failure{PRIMA_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path};
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    std::string base(path);
    const size_t slash = base.find_last_of('/');
    if (slash != std::string::npos) base = base.substr(slash + 1);
    auto h = std::make_unique<prima_mps_instance>();
    h->inst = prima::model::read_text(text.data(), (int64_t)text.size(), base);
    *out = h.release();
  });
}

extern "C" void prima_mps_free(prima_mps_instance *mps) { delete mps; }

extern "C" int32_t prima_mps_get_info(const prima_mps_instance *mps, prima_mps_info *info) {
  return guarded([&] {
    if (!mps || !info) require_fail("mps or info is NULL");
    const auto &I = mps->inst;
    info->num_variables = I.lp.n;
    info->num_constraints = I.lp.m;
    info->num_equalities = I.lp.neq;
    info->num_rows = (int32_t)I.row_names.size();
    info->nnz = (int64_t)I.lp.ci.size();
    info->num_integer_columns = (int32_t)I.integer_cols.size();
    info->pad = 0;
  });
}

extern "C" int32_t prima_mps_get_problem(const prima_mps_instance *mps, prima_lp *lp) {
  return guarded([&] {
    if (!mps || !lp) require_fail("mps or lp is NULL");
    *lp = mps->inst.lp.view();
  });
}

extern "C" int32_t prima_mps_get_translation(const prima_mps_instance *mps, int32_t *kind, int32_t *first,
                                             int32_t *second) {
  return guarded([&] {
    if (!mps || !kind || !first || !second) require_fail("NULL argument");
    const auto &I = mps->inst;
    std::copy(I.kind.begin(), I.kind.end(), kind);
    std::copy(I.first.begin(), I.first.end(), first);
    std::copy(I.second.begin(), I.second.end(), second);
  });
}

extern "C" const char *prima_mps_name(const prima_mps_instance *mps) { return mps ? mps->inst.name.c_str() : ""; }

extern "C" const char *prima_mps_row_name(const prima_mps_instance *mps, int32_t row) {
  if (!mps || row < 0 || (size_t)row >= mps->inst.row_names.size()) return nullptr;
  return mps->inst.row_names[(size_t)row].c_str();
}

extern "C" const char *prima_mps_column_name(const prima_mps_instance *mps, int32_t column) {
  if (!mps || column < 0 || (size_t)column >= mps->inst.col_names.size()) return nullptr;
  return mps->inst.col_names[(size_t)column].c_str();
}

extern "C" int32_t prima_mps_get_integer_columns(const prima_mps_instance *mps, int32_t *columns) {
  return guarded([&] {
    if (!mps || !columns) require_fail("NULL argument");
    std::copy(mps->inst.integer_cols.begin(), mps->inst.integer_cols.end(), columns);
  });
}

extern "C" int32_t prima_presolve(const prima_lp *lp, int32_t max_passes, prima_presolved **out) {
  return guarded([&] {
    if (!out) require_fail("out is NULL");
    *out = nullptr;
    if (max_passes < 0) require_fail("max_passes must be non-negative");
    auto h = std::make_unique<prima_presolved>();
    h->p.original = prima::model::copy_lp(lp);
    prima::model::presolve(h->p, max_passes);
    *out = h.release();
  });
}

extern "C" void prima_presolve_free(prima_presolved *presolved) { delete presolved; }

extern "C" int32_t prima_presolve_get_info(const prima_presolved *presolved, prima_presolve_info *info) {
  return guarded([&] {
    if (!presolved || !info) require_fail("presolved or info is NULL");
    const auto &P = presolved->p;
    info->fixed_columns = P.fixed;
    info->empty_columns = P.empty_cols;
    info->empty_rows = P.empty_rows;
    info->singleton_rows = P.singletons;
    info->proven_infeasible = P.infeasible;
    info->unbounded_if_feasible = P.unbounded_if_feasible;
    info->passes = P.passes;
    info->reduced_variables = P.infeasible ? 0 : P.reduced.n;
    info->reduced_constraints = P.infeasible ? 0 : P.reduced.m;
    info->reduced_equalities = P.infeasible ? 0 : P.reduced.neq;
    info->reduced_nnz = P.infeasible ? 0 : (int64_t)P.reduced.ci.size();
  });
}

extern "C" int32_t prima_presolve_get_reduced(const prima_presolved *presolved, prima_lp *reduced) {
  return guarded([&] {
    if (!presolved || !reduced) require_fail("presolved or reduced is NULL");
    if (presolved->p.infeasible)
      require_fail("presolve already established PRIMAL_INFEASIBLE; there is nothing to solve");
    *reduced = presolved->p.reduced.view();
  });
}

extern "C" int32_t prima_presolve_get_maps(const prima_presolved *presolved, int32_t *column_map, int32_t *row_map) {
  return guarded([&] {
    if (!presolved || !column_map || !row_map) require_fail("NULL argument");
    const auto &P = presolved->p;
    std::copy(P.column_map.begin(), P.column_map.end(), column_map);
    std::copy(P.row_map.begin(), P.row_map.end(), row_map);
  });
}

extern "C" int32_t prima_presolve_restore(const prima_presolved *presolved, const double *primal, const double *dual,
                                          const double *reduced_costs, double *primal_out, double *dual_out,
                                          double *reduced_costs_out) {
  return guarded([&] {
    if (!presolved) require_fail("presolved is NULL");
    const auto &P = presolved->p;
    if (P.infeasible)
      require_fail("presolve already established PRIMAL_INFEASIBLE; restoring a reduced solution would fabricate one");
    if ((!primal && !P.column_map.empty()) || (!reduced_costs && !P.column_map.empty()) ||
        (!dual && !P.row_map.empty()) || !primal_out || !dual_out || !reduced_costs_out)
      require_fail("NULL argument");
    prima::model::restore(P, primal, dual, reduced_costs, primal_out, dual_out, reduced_costs_out);
  });
}
