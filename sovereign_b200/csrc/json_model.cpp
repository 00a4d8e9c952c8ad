// json_model.cpp -- the reference's JSON model format read straight into the index form of
// sov_model (column-compressed A, per-variable arrays), without name-keyed maps.
//
// Format (solver/core/src/json_io.cpp:13-80): {"problem_type": "LP"|"QP"|"MILP", "sense":
// "minimize"|"maximize" (default minimize), "variables": [{"name", "type" (default continuous),
// "lower_bound" (default 0; binary 0), "upper_bound" (default 1e30; binary 1)}], "objective":
// {"constant", "linear": {name: value}, "quadratic": {name: {name: value}}}, "constraints":
// [{"name" (default ""), "sense": "<=" | ">=" | "=" (and the aliases of types.cpp:97-102), "rhs",
// "linear": {name: value}}]}. Keys may come in any order and unknown keys are skipped.
//
// The reference parses the whole document into a DOM, then into hash maps keyed by name, and the
// IPM turns those maps back into a sparse matrix (interior_point.cpp:224-409); on large models that
// load dominates the run. Here one pass over the text records every term as (row, name span,
// value), names are resolved through one hash table of the variables, and a counting sort by column
// builds A directly: rows come out ascending within each column, as the adapter's conversion gives
// them. Unknown variables in a constraint are rejected with the IPM's own message ("Unknown variable
// in constraint: <name>"); objective and quadratic terms on unknown names are ignored, as the
// IPM's conversion ignores them.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "errors.hpp"
#include "sov_ipm.h"

struct sov_json_model {
  int32_t problem_type = 0;  // 0 LP, 1 QP, 2 MILP (types.hpp ProblemType order)
  std::vector<std::string> var_names, row_names;
  std::vector<int8_t> var_type;  // 0 continuous, 1 integer, 2 binary
  std::vector<int32_t> col_ptr, row_idx, q_col_ptr, q_row_idx;
  std::vector<double> values, obj, lb, ub, rhs, q_values;
  std::vector<int8_t> sense;
  sov_model view{};
};

namespace {

class Reader {
 public:
  Reader(const char* p, size_t n) : p_(p), e_(p + n) {}

  [[noreturn]] void fail(const std::string& what) const {
    throw std::invalid_argument("JSON model: " + what + " at byte " + std::to_string(p_ - begin_));
  }
  void set_begin(const char* b) { begin_ = b; }
  void ws() {
    while (p_ < e_ && (*p_ == ' ' || *p_ == '\n' || *p_ == '\r' || *p_ == '\t')) ++p_;
  }
  bool peek(char c) {
    ws();
    return p_ < e_ && *p_ == c;
  }
  void expect(char c) {
    ws();
    if (p_ >= e_ || *p_ != c) fail(std::string("expected '") + c + "'");
    ++p_;
  }
  bool eat(char c) {
    if (peek(c)) {
      ++p_;
      return true;
    }
    return false;
  }
  // A string: the raw span when it has no escapes, else the decoded copy in `scratch`.
  std::string_view string(std::string& scratch) {
    expect('"');
    const char* s = p_;
    while (p_ < e_ && *p_ != '"' && *p_ != '\\') ++p_;
    if (p_ < e_ && *p_ == '"') return std::string_view(s, static_cast<size_t>(p_++ - s));
    scratch.assign(s, p_);
    while (p_ < e_ && *p_ != '"') {
      if (*p_ != '\\') {
        scratch.push_back(*p_++);
        continue;
      }
      if (++p_ >= e_) break;
      const char c = *p_++;
      switch (c) {
        case 'n': scratch.push_back('\n'); break;
        case 't': scratch.push_back('\t'); break;
        case 'r': scratch.push_back('\r'); break;
        case 'b': scratch.push_back('\b'); break;
        case 'f': scratch.push_back('\f'); break;
        case 'u': {
          if (e_ - p_ < 4) fail("short \\u escape");
          unsigned cp = 0;
          for (int k = 0; k < 4; ++k) {
            const char h = *p_++;
            cp = cp * 16 + static_cast<unsigned>(h >= '0' && h <= '9' ? h - '0' : h >= 'a' && h <= 'f' ? h - 'a' + 10
                                                  : h >= 'A' && h <= 'F' ? h - 'A' + 10 : (fail("bad \\u escape"), 0));
          }
          if (cp >= 0xD800 && cp < 0xDC00 && e_ - p_ >= 6 && p_[0] == '\\' && p_[1] == 'u') {  // surrogate pair
            unsigned lo = 0;
            for (int k = 2; k < 6; ++k) {
              const char h = p_[k];
              lo = lo * 16 + static_cast<unsigned>(h >= '0' && h <= '9' ? h - '0' : h >= 'a' && h <= 'f' ? h - 'a' + 10
                                                   : h >= 'A' && h <= 'F' ? h - 'A' + 10 : 0);
            }
            if (lo >= 0xDC00 && lo < 0xE000) {
              cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
              p_ += 6;
            }
          }
          if (cp < 0x80) {
            scratch.push_back(static_cast<char>(cp));
          } else if (cp < 0x800) {
            scratch.push_back(static_cast<char>(0xC0 | (cp >> 6)));
            scratch.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
          } else if (cp < 0x10000) {
            scratch.push_back(static_cast<char>(0xE0 | (cp >> 12)));
            scratch.push_back(static_cast<char>(0x80 | ((cp >> 6) & 0x3F)));
            scratch.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
          } else {
            scratch.push_back(static_cast<char>(0xF0 | (cp >> 18)));
            scratch.push_back(static_cast<char>(0x80 | ((cp >> 12) & 0x3F)));
            scratch.push_back(static_cast<char>(0x80 | ((cp >> 6) & 0x3F)));
            scratch.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
          }
          break;
        }
        default: scratch.push_back(c);  // \" \\ \/
      }
    }
    if (p_ >= e_) fail("unterminated string");
    ++p_;
    return scratch;
  }
  double number() {
    ws();
    double v = 0.0;
    const char* s = p_;
    if (s < e_ && *s == '+') fail("bad number");
    const auto r = std::from_chars(s, e_, v);
    if (r.ec == std::errc::result_out_of_range) {  // beyond the FP64 range: +-inf, or a signed zero
      const std::string_view text(s, static_cast<size_t>(r.ptr - s));
      const size_t ep = text.find_first_of("eE");
      const bool tiny = ep != std::string_view::npos && ep + 1 < text.size() && text[ep + 1] == '-';
      const bool neg = !text.empty() && text[0] == '-';
      p_ = r.ptr;
      return tiny ? (neg ? -0.0 : 0.0) : (neg ? -HUGE_VAL : HUGE_VAL);
    }
    if (r.ec != std::errc()) fail("bad number");
    p_ = r.ptr;
    return v;
  }
  // skips any value
  void skip() {
    ws();
    if (p_ >= e_) fail("unexpected end");
    std::string scratch;
    switch (*p_) {
      case '"': string(scratch); return;
      case '{':
        ++p_;
        if (eat('}')) return;
        do {
          string(scratch);
          expect(':');
          skip();
        } while (eat(','));
        expect('}');
        return;
      case '[':
        ++p_;
        if (eat(']')) return;
        do skip();
        while (eat(','));
        expect(']');
        return;
      case 't': literal("true"); return;
      case 'f': literal("false"); return;
      case 'n': literal("null"); return;
      default: number();
    }
  }
  void literal(const char* w) {
    const size_t k = std::strlen(w);
    if (static_cast<size_t>(e_ - p_) < k || std::memcmp(p_, w, k) != 0) fail("bad literal");
    p_ += k;
  }
  // iterate the members of an object: fn(key) must consume the value
  template <class F>
  void object(F&& fn) {
    expect('{');
    if (eat('}')) return;
    std::string scratch;
    do {
      const std::string_view key = string(scratch);
      const std::string k(key);
      expect(':');
      fn(k);
    } while (eat(','));
    expect('}');
  }
  template <class F>
  void array(F&& fn) {
    expect('[');
    if (eat(']')) return;
    do fn();
    while (eat(','));
    expect(']');
  }
  bool at_end() {
    ws();
    return p_ >= e_;
  }

 private:
  const char* p_;
  const char* e_;
  const char* begin_ = nullptr;
};

struct Term {
  int32_t row;
  uint32_t name;  // index into the name pool
  double value;
};

int8_t constraint_sense(const std::string& s) {
  if (s == "<=" || s == "le" || s == "LE") return SOV_LE;
  if (s == ">=" || s == "ge" || s == "GE") return SOV_GE;
  if (s == "=" || s == "==" || s == "eq" || s == "EQ") return SOV_EQ;
  throw std::invalid_argument("Unknown constraint sense: " + s);
}

void parse(const char* text, size_t len, sov_json_model& jm) {
  Reader rd(text, len);
  rd.set_begin(text);
  std::vector<std::string> pool;  // term names (copied: keys may be decoded escapes)
  std::unordered_map<std::string, uint32_t> pool_index;
  auto intern = [&](std::string_view s) {
    auto it = pool_index.find(std::string(s));
    if (it != pool_index.end()) return it->second;
    const uint32_t id = static_cast<uint32_t>(pool.size());
    pool.emplace_back(s);
    pool_index.emplace(pool.back(), id);
    return id;
  };
  std::vector<Term> terms;                      // constraint terms, row order
  std::vector<std::pair<uint32_t, double>> lin;  // objective linear terms
  struct QTerm {
    uint32_t row, col;
    double value;
  };
  std::vector<QTerm> quad;
  bool have_type = false, maximize = false;
  double constant = 0.0;
  int rows = 0;
  rd.object([&](const std::string& key) {
    std::string scratch;
    if (key == "problem_type") {
      const std::string t(rd.string(scratch));
      if (t == "LP" || t == "lp") jm.problem_type = 0;
      else if (t == "QP" || t == "qp") jm.problem_type = 1;
      else if (t == "MILP" || t == "milp") jm.problem_type = 2;
      else throw std::invalid_argument("Unknown problem_type: " + t);
      have_type = true;
    } else if (key == "sense") {
      const std::string t(rd.string(scratch));
      if (t == "minimize" || t == "min") maximize = false;
      else if (t == "maximize" || t == "max") maximize = true;
      else throw std::invalid_argument("Unknown sense: " + t);
    } else if (key == "variables") {
      rd.array([&]() {
        std::string name;
        bool has_name = false, has_lb = false, has_ub = false;
        int8_t type = 0;
        double lo = 0.0, hi = 1e30;
        rd.object([&](const std::string& k) {
          std::string sc;
          if (k == "name") {
            name = std::string(rd.string(sc));
            has_name = true;
          } else if (k == "type") {
            const std::string t(rd.string(sc));
            if (t == "continuous") type = 0;
            else if (t == "integer") type = 1;
            else if (t == "binary") type = 2;
            else throw std::invalid_argument("Unknown variable type: " + t);
          } else if (k == "lower_bound") {
            lo = rd.number();
            has_lb = true;
          } else if (k == "upper_bound") {
            hi = rd.number();
            has_ub = true;
          } else {
            rd.skip();
          }
        });
        if (!has_name) throw std::invalid_argument("JSON model: a variable has no name");
        if (type == 2) {  // binary defaults (json_io.cpp:26-29)
          if (!has_lb) lo = 0.0;
          if (!has_ub) hi = 1.0;
        }
        jm.var_names.push_back(std::move(name));
        jm.var_type.push_back(type);
        jm.lb.push_back(lo);
        jm.ub.push_back(hi);
      });
    } else if (key == "objective") {
      rd.object([&](const std::string& k) {
        if (k == "constant") {
          constant = rd.number();
        } else if (k == "linear") {
          rd.object([&](const std::string& name) { lin.push_back({intern(name), rd.number()}); });
        } else if (k == "quadratic") {
          rd.object([&](const std::string& rname) {
            const uint32_t r = intern(rname);
            rd.object([&](const std::string& cname) { quad.push_back({r, intern(cname), rd.number()}); });
          });
        } else {
          rd.skip();
        }
      });
    } else if (key == "constraints") {
      rd.array([&]() {
        std::string name;
        bool has_sense = false, has_rhs = false;
        int8_t s = SOV_EQ;
        double b = 0.0;
        const int row = rows++;
        rd.object([&](const std::string& k) {
          std::string sc;
          if (k == "name") {
            name = std::string(rd.string(sc));
          } else if (k == "sense") {
            s = constraint_sense(std::string(rd.string(sc)));
            has_sense = true;
          } else if (k == "rhs") {
            b = rd.number();
            has_rhs = true;
          } else if (k == "linear") {
            rd.object([&](const std::string& v) { terms.push_back({row, intern(v), rd.number()}); });
          } else {
            rd.skip();
          }
        });
        if (!has_sense || !has_rhs) throw std::invalid_argument("JSON model: constraint without sense or rhs");
        jm.row_names.push_back(std::move(name));
        jm.sense.push_back(s);
        jm.rhs.push_back(b);
      });
    } else {
      rd.skip();
    }
  });
  if (!rd.at_end()) rd.fail("trailing characters");
  if (!have_type) throw std::invalid_argument("JSON model: no problem_type");
  const int n = static_cast<int>(jm.var_names.size());
  // names -> columns (a repeated variable name resolves to its last column, as the name index of
  // the IPM's conversion does)
  std::unordered_map<std::string_view, int32_t> col_of;
  col_of.reserve(static_cast<size_t>(n) * 2);
  for (int j = 0; j < n; ++j) col_of[jm.var_names[j]] = j;
  std::vector<int32_t> pool_col(pool.size(), -1);
  for (size_t k = 0; k < pool.size(); ++k) {
    auto it = col_of.find(pool[k]);
    if (it != col_of.end()) pool_col[k] = it->second;
  }
  jm.obj.assign(n, 0.0);
  for (const auto& t : lin)
    if (pool_col[t.first] >= 0) jm.obj[pool_col[t.first]] = t.second;  // a repeated key: the last one
  // A by counting sort on the column; terms are in row order, so rows ascend within a column
  jm.col_ptr.assign(n + 1, 0);
  for (const Term& t : terms) {
    const int32_t j = pool_col[t.name];
    if (j < 0) throw std::invalid_argument("Unknown variable in constraint: " + pool[t.name]);
    jm.col_ptr[j + 1]++;
  }
  for (int j = 0; j < n; ++j) jm.col_ptr[j + 1] += jm.col_ptr[j];
  jm.row_idx.resize(terms.size());
  jm.values.resize(terms.size());
  {
    std::vector<int32_t> at(jm.col_ptr.begin(), jm.col_ptr.end() - 1);
    for (const Term& t : terms) {
      const int32_t j = pool_col[t.name];
      jm.row_idx[at[j]] = t.row;
      jm.values[at[j]++] = t.value;
    }
  }
  if (!quad.empty()) {  // stored terms q_ij, column-compressed by j = the inner name
    jm.q_col_ptr.assign(n + 1, 0);
    std::vector<std::pair<int32_t, int32_t>> ij;
    for (const auto& t : quad) {
      const int32_t i = pool_col[t.row], j = pool_col[t.col];
      if (i >= 0 && j >= 0) jm.q_col_ptr[j + 1]++;
    }
    for (int j = 0; j < n; ++j) jm.q_col_ptr[j + 1] += jm.q_col_ptr[j];
    jm.q_row_idx.resize(jm.q_col_ptr[n]);
    jm.q_values.resize(jm.q_col_ptr[n]);
    std::vector<int32_t> at(jm.q_col_ptr.begin(), jm.q_col_ptr.end() - 1);
    for (const auto& t : quad) {
      const int32_t i = pool_col[t.row], j = pool_col[t.col];
      if (i < 0 || j < 0) continue;
      jm.q_row_idx[at[j]] = i;
      jm.q_values[at[j]++] = t.value;
    }
  }
  sov_model& v = jm.view;
  v.n = n;
  v.m = rows;
  v.maximize = maximize ? 1 : 0;
  v.col_ptr = jm.col_ptr.data();
  v.row_idx = jm.row_idx.data();
  v.values = jm.values.data();
  v.obj = jm.obj.data();
  v.obj_constant = constant;
  v.lb = jm.lb.data();
  v.ub = jm.ub.data();
  v.sense = jm.sense.data();
  v.rhs = jm.rhs.data();
  if (!quad.empty()) {
    v.q_col_ptr = jm.q_col_ptr.data();
    v.q_row_idx = jm.q_row_idx.data();
    v.q_values = jm.q_values.data();
  }
}

}  // namespace

extern "C" {

int sov_model_from_json(const char* text, size_t len, sov_json_model** out) {
  if (!text || !out) return sov::record_error(SOV_E_ARGUMENT, "JSON model: null text or output");
  *out = nullptr;
  auto* jm = new (std::nothrow) sov_json_model();
  if (!jm) return sov::record_error(SOV_E_ARGUMENT, "JSON model: out of host memory");
  try {
    parse(text, len, *jm);
  } catch (const std::exception& e) {
    delete jm;
    return sov::record_error(SOV_E_ARGUMENT, e.what());
  }
  *out = jm;
  return SOV_OK;
}

const sov_model* sov_json_model_view(const sov_json_model* jm) { return jm ? &jm->view : nullptr; }

int32_t sov_json_model_problem_type(const sov_json_model* jm) { return jm ? jm->problem_type : -1; }

int32_t sov_json_model_variable_type(const sov_json_model* jm, int32_t j) {
  return jm && j >= 0 && j < static_cast<int32_t>(jm->var_type.size()) ? jm->var_type[j] : -1;
}

const char* sov_json_model_variable_name(const sov_json_model* jm, int32_t j) {
  return jm && j >= 0 && j < static_cast<int32_t>(jm->var_names.size()) ? jm->var_names[j].c_str() : nullptr;
}

const char* sov_json_model_row_name(const sov_json_model* jm, int32_t i) {
  return jm && i >= 0 && i < static_cast<int32_t>(jm->row_names.size()) ? jm->row_names[i].c_str() : nullptr;
}

void sov_json_model_destroy(sov_json_model* jm) { delete jm; }

}  // extern "C"
