// The dense normal-matrix gather map (build_assembly_dense: per-row bucketing, no global sort)
// against the generic sort-based builder in row-major order (build_assembly_rowmajor): every
// lower-triangle target must receive the same contributions (column, weight bit for bit) in the
// same order, so the gather sums identically. Also with the row-wise copy absent from the form
// (the dense builder then makes its own) and with empty rows (diagonal targets without entries).
#include <cstdio>
#include <cstring>
#include <map>
#include <random>
#include <vector>

#include "stdform.hpp"

using namespace sov;

namespace {

int compare(const AssemblyMap& dense, const AssemblyMap& rowmajor, int m, int ld) {
  std::map<int64_t, int> by_target;  // row-major target -> its index
  for (std::size_t t = 0; t < rowmajor.target.size(); ++t) by_target[rowmajor.target[t]] = static_cast<int>(t);
  int bad = 0;
  if (dense.target.size() != rowmajor.target.size()) return 1;
  for (std::size_t t = 0; t < dense.target.size(); ++t) {
    if (t > 0 && dense.target[t] <= dense.target[t - 1]) ++bad;  // sorted, distinct
    const int64_t c = dense.target[t] / ld, r = dense.target[t] % ld;
    if (r < c) ++bad;
    const auto it = by_target.find(r * ld + c);
    if (it == by_target.end()) {
      ++bad;
      continue;
    }
    const int u = it->second;
    const int n1 = dense.ptr[t + 1] - dense.ptr[t], n2 = rowmajor.ptr[u + 1] - rowmajor.ptr[u];
    if (n1 != n2) {
      ++bad;
      continue;
    }
    for (int k = 0; k < n1; ++k) {
      if (dense.col[dense.ptr[t] + k] != rowmajor.col[rowmajor.ptr[u] + k]) ++bad;
      if (std::memcmp(&dense.w[dense.ptr[t] + k], &rowmajor.w[rowmajor.ptr[u] + k], sizeof(double)) != 0) ++bad;
    }
  }
  for (int i = 0; i < m; ++i) {
    const int t = dense.diag_target[i];
    if (t < 0 || dense.target[t] != static_cast<int64_t>(i) * ld + i) ++bad;
  }
  return bad;
}

}  // namespace

int main() {
  std::mt19937 rng(11);
  int bad = 0, tested = 0;
  for (int t = 0; t < 400; ++t) {
    const int m = 1 + rng() % 60, n = 1 + rng() % 120;
    const int density = 2 + rng() % 6;
    std::vector<int> cp(1, 0), ri;
    std::vector<double> v, c(n), lb(n, 0.0), ub(n, 1e30), rhs(m);
    std::vector<int8_t> sense(m);
    const int empty_row = (t % 3 == 0) ? static_cast<int>(rng() % m) : -1;
    for (int j = 0; j < n; ++j) {
      for (int r = 0; r < m; ++r)
        if (r != empty_row && rng() % density == 0) {
          ri.push_back(r);
          v.push_back((int(rng() % 2001) - 1000) / 37.0);
        }
      cp.push_back(static_cast<int>(ri.size()));
      c[j] = (int(rng() % 200) - 100) / 3.0;
      if (rng() % 4 == 0) ub[j] = (rng() % 100) / 3.0;
    }
    for (int r = 0; r < m; ++r) {
      rhs[r] = (int(rng() % 1000) - 500) / 11.0;
      sense[r] = static_cast<int8_t>(rng() % 3);
    }
    sov_model p{};
    p.n = n;
    p.m = m;
    p.col_ptr = cp.data();
    p.row_idx = ri.data();
    p.values = v.data();
    p.obj = c.data();
    p.lb = lb.data();
    p.ub = ub.data();
    p.sense = sense.data();
    p.rhs = rhs.data();
    const StdForm f = build_std_form(p, false, t % 2 == 0);
    const int ld = (f.m + 63) / 64 * 64;
    const AssemblyMap ref = build_assembly_rowmajor(f, ld);
    bad += compare(build_assembly_dense(f, ld), ref, f.m, ld);
    StdForm bare = f;  // no row-wise copy
    bare.row_ptr.clear();
    bare.col_idx.clear();
    bare.rval.clear();
    bad += compare(build_assembly_dense(bare, ld), ref, f.m, ld);
    ++tested;
  }
  std::printf("tested %d mismatches %d\n", tested, bad);
  return bad == 0 ? 0 : 1;
}
