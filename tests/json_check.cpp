// The CSC-native JSON ingest (sov_model_from_json) against the reference's own reader
// (solver/core/src/json_io.cpp load_model_from_json_string) followed by the index conversion the
// IPM adapter applies (include/sov_ipm_adapter.hpp detail::to_index): n, m, sense, A (column
// pointers, rows, values bit for bit), objective, bounds, row senses and right-hand sides, Q terms
// and the constant must be identical, and so must the error message of a model that names an
// unknown variable. Each JSON file given on the command line is checked, and the ingest of the
// largest is timed against the reference's. Prints "failures N". Built by oracle/Makefile with the
// reference library (it compiles the reference's reader); CPU only.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "sov_ipm_adapter.hpp"
#include "sovereign/json_io.hpp"

using namespace sovereign;

namespace {

int failures = 0;

template <class T>
bool same(const T* a, const T* b, int n) {
  return n == 0 || std::memcmp(a, b, sizeof(T) * static_cast<size_t>(n)) == 0;
}

void check(const std::string& name, const std::string& text) {
  sov_json_model* jm = nullptr;
  const int rc = sov_model_from_json(text.data(), text.size(), &jm);
  std::string ref_error;
  OptimizationModel ref;
  b200::detail::IndexModel im;
  try {
    ref = load_model_from_json_string(text);
    im = b200::detail::to_index(ref, ref.problem_type == ProblemType::QP);
  } catch (const std::exception& e) {
    ref_error = e.what();
  }
  if (!ref_error.empty()) {
    const std::string got = rc == SOV_OK ? "" : sov_last_error();
    if (rc == SOV_OK || got.find(ref_error) == std::string::npos) {
      std::printf("FAIL %s: reference error '%s', ingest '%s'\n", name.c_str(), ref_error.c_str(), got.c_str());
      ++failures;
    } else {
      std::printf("ok %s: both refuse (%s)\n", name.c_str(), ref_error.c_str());
    }
    if (jm) sov_json_model_destroy(jm);
    return;
  }
  if (rc != SOV_OK) {
    std::printf("FAIL %s: ingest refused: %s\n", name.c_str(), sov_last_error());
    ++failures;
    return;
  }
  const sov_model& a = *sov_json_model_view(jm);
  const sov_model& b = im.view;
  const int nnz = b.col_ptr[b.n];
  bool ok = a.n == b.n && a.m == b.m && a.maximize == b.maximize && a.obj_constant == b.obj_constant &&
            same(a.col_ptr, b.col_ptr, b.n + 1) && a.col_ptr[a.n] == nnz && same(a.row_idx, b.row_idx, nnz) &&
            same(a.values, b.values, nnz) && same(a.obj, b.obj, b.n) && same(a.lb, b.lb, b.n) &&
            same(a.ub, b.ub, b.n) && same(a.sense, b.sense, b.m) && same(a.rhs, b.rhs, b.m) &&
            sov_json_model_problem_type(jm) == static_cast<int>(ref.problem_type);
  for (int j = 0; ok && j < b.n; ++j) ok = ref.variables[j].name == sov_json_model_variable_name(jm, j) &&
                                          static_cast<int>(ref.variables[j].type) == sov_json_model_variable_type(jm, j);
  for (int i = 0; ok && i < b.m; ++i) ok = ref.constraints[i].name == sov_json_model_row_name(jm, i);
  if (ok && b.q_col_ptr) {
    // stored Q terms: the same multiset per column (the reference's maps give no order)
    ok = a.q_col_ptr && same(a.q_col_ptr, b.q_col_ptr, b.n + 1);
    for (int j = 0; ok && j < b.n; ++j) {
      std::vector<std::pair<int, double>> x, y;
      for (int k = a.q_col_ptr[j]; k < a.q_col_ptr[j + 1]; ++k) x.push_back({a.q_row_idx[k], a.q_values[k]});
      for (int k = b.q_col_ptr[j]; k < b.q_col_ptr[j + 1]; ++k) y.push_back({b.q_row_idx[k], b.q_values[k]});
      std::sort(x.begin(), x.end());
      std::sort(y.begin(), y.end());
      ok = x == y;
    }
  } else if (ok) {
    ok = a.q_col_ptr == nullptr;
  }
  std::printf("%s %s: n=%d m=%d nnz=%d\n", ok ? "ok" : "FAIL", name.c_str(), b.n, b.m, nnz);
  if (!ok) ++failures;
  sov_json_model_destroy(jm);
}

std::string read(const char* path) {
  std::ifstream in(path, std::ios::binary);
  std::stringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

}  // namespace

int main(int argc, char** argv) {
  std::string largest;
  for (int k = 1; k < argc; ++k) {
    const std::string text = read(argv[k]);
    check(argv[k], text);
    if (text.size() > largest.size()) largest = text;
  }
  // generated cases: keys out of order, escapes, defaults, binary bounds, QP terms, maximisation,
  // unknown keys, an unknown variable
  check("keys out of order",
        R"({"constraints": [{"linear": {"b": 2.5, "a": -1}, "rhs": 3, "sense": ">=", "name": "r0"},
             {"sense": "=", "rhs": 1e-3, "linear": {"a": 1}}],
            "objective": {"linear": {"a": 1.25, "b": -2, "zz": 7}, "constant": 4.5},
            "extra": [1, {"x": null}, true, "s"], "sense": "max",
            "variables": [{"name": "a", "upper_bound": 10}, {"type": "binary", "name": "b"},
                          {"name": "c", "lower_bound": -1e30, "type": "integer"}], "problem_type": "lp"})");
  check("escaped names", R"({"problem_type": "LP", "variables": [{"name": "x\"1"}, {"name": "yé\\z"}],
            "objective": {"linear": {"x\"1": 1, "yé\\z": 2}},
            "constraints": [{"name": "c\n1", "sense": "le", "rhs": 4, "linear": {"yé\\z": 1, "x\"1": 1}}]})");
  check("quadratic", R"({"problem_type": "QP", "sense": "minimize",
            "variables": [{"name": "p", "lower_bound": -1e30}, {"name": "q"}, {"name": "r"}],
            "objective": {"linear": {"p": -1}, "quadratic": {"p": {"p": 2, "q": 0.5}, "r": {"q": 1, "r": 3}}},
            "constraints": [{"sense": "<=", "rhs": 1, "linear": {"p": 1, "q": 1, "r": 1}}]})");
  check("unknown variable", R"({"problem_type": "LP", "variables": [{"name": "a"}],
            "constraints": [{"sense": "<=", "rhs": 1, "linear": {"a": 1, "nope": 2}}]})");
  check("empty", R"({"problem_type": "LP", "variables": []})");
  if (!largest.empty()) {  // ingest time of the largest file: the reference's path against this one
    const auto t0 = std::chrono::steady_clock::now();
    const OptimizationModel ref = load_model_from_json_string(largest);
    const b200::detail::IndexModel im = b200::detail::to_index(ref, false);
    const auto t1 = std::chrono::steady_clock::now();
    sov_json_model* jm = nullptr;
    sov_model_from_json(largest.data(), largest.size(), &jm);
    const auto t2 = std::chrono::steady_clock::now();
    std::printf("ingest of %zu bytes: reference reader + index conversion %.1f ms, CSC-native %.1f ms\n",
                largest.size(), 1e3 * std::chrono::duration<double>(t1 - t0).count(),
                1e3 * std::chrono::duration<double>(t2 - t1).count());
    sov_json_model_destroy(jm);
  }
  std::printf("failures %d\n", failures);
  return failures == 0 ? 0 : 1;
}
