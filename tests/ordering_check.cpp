// The host ordering and symbolic analysis of the sparse L D L' (sovereign_b200/csrc/sparse.cpp),
// without a GPU: on grid-network and random normal-matrix patterns the ordering must be a
// permutation, the column patterns of L must equal a brute-force symbolic elimination of
// A A' in that order, the elimination tree must be the first off-diagonal row of each column,
// the level schedule must cover every column once with children below their parents, and the fill
// on the 130 x 130 grid must stay near the reference's nnz(L) = 409164. Prints "failures 0".
#include <chrono>
#include <cstdio>
#include <random>
#include <set>
#include <vector>

#include "sparse.hpp"

using namespace sov;

static StdForm from_columns(int m, const std::vector<std::vector<int>>& cols) {
  StdForm f;
  f.m = m;
  f.n = static_cast<int>(cols.size());
  f.col_ptr.push_back(0);
  for (const auto& c : cols) {
    for (int r : c) {
      f.row_idx.push_back(r);
      f.val.push_back(1.0);
    }
    f.col_ptr.push_back(static_cast<int>(f.row_idx.size()));
  }
  return f;
}

static StdForm grid(int g) {  // arcs of a g x g grid: every column touches two adjacent nodes
  std::vector<std::vector<int>> cols;
  for (int i = 0; i < g; ++i)
    for (int j = 0; j < g; ++j) {
      const int a = i * g + j;
      if (i + 1 < g) cols.push_back({a, a + g});
      if (j + 1 < g) cols.push_back({a, a + 1});
    }
  return from_columns(g * g, cols);
}

static StdForm random_pattern(int m, int n, int k, unsigned seed) {
  std::mt19937 rng(seed);
  std::vector<std::vector<int>> cols(n);
  for (auto& c : cols) {
    std::set<int> rows;
    while (static_cast<int>(rows.size()) < k) rows.insert(static_cast<int>(rng() % m));
    c.assign(rows.begin(), rows.end());
  }
  return from_columns(m, cols);
}

// brute force: eliminate in the given order on an explicit adjacency matrix
static long long check(const StdForm& f, const SparseSymbolic& s, const char* name) {
  const int m = f.m;
  long long bad = 0;
  std::vector<int> seen(m, 0);
  for (int k = 0; k < m; ++k) {
    if (s.perm[k] < 0 || s.perm[k] >= m || seen[s.perm[k]]++) ++bad;
    if (s.iperm[s.perm[k]] != k) ++bad;
  }
  if (bad) {
    std::printf("%s: not a permutation\n", name);
    return bad;
  }
  std::vector<std::set<int>> g(m);  // permuted indices
  for (int j = 0; j < f.n; ++j)
    for (int p = f.col_ptr[j]; p < f.col_ptr[j + 1]; ++p)
      for (int q = f.col_ptr[j]; q < f.col_ptr[j + 1]; ++q)
        if (p != q) g[s.iperm[f.row_idx[p]]].insert(s.iperm[f.row_idx[q]]);
  for (int k = 0; k < m; ++k) {
    std::vector<int> below;
    for (int i : g[k])
      if (i > k) below.push_back(i);
    const std::vector<int> got(s.li.begin() + s.lp[k], s.li.begin() + s.lp[k + 1]);
    if (got != below) ++bad;
    if (s.parent[k] != (below.empty() ? -1 : below.front())) ++bad;
    for (int a : below)
      for (int b : below)
        if (a != b) g[a].insert(b);
  }
  std::vector<int> level_of(m, -1);
  for (int h = 0; h < s.levels(); ++h)
    for (int q = s.lvl_ptr[h]; q < s.lvl_ptr[h + 1]; ++q) {
      if (level_of[s.lvl_col[q]] >= 0) ++bad;
      level_of[s.lvl_col[q]] = h;
    }
  for (int k = 0; k < m; ++k)
    if (level_of[k] < 0 || (s.parent[k] >= 0 && level_of[s.parent[k]] <= level_of[k])) ++bad;
  std::printf("%s: m=%d nnz(L)=%lld levels=%d mismatches=%lld\n", name, m, s.nnz_l, s.levels(), bad);
  return bad;
}

int main() {
  long long failures = 0;
  struct Case {
    const char* name;
    StdForm f;
  };
  std::vector<Case> cases;
  cases.push_back({"grid 12x12", grid(12)});
  cases.push_back({"grid 30x30", grid(30)});
  cases.push_back({"random 200x1000 k=3", random_pattern(200, 1000, 3, 1)});
  cases.push_back({"random 300x600 k=2", random_pattern(300, 600, 2, 2)});
  cases.push_back({"random 150x400 k=6 (dense rows held back)", random_pattern(150, 400, 6, 3)});
  cases.push_back({"random 1x5 k=1", random_pattern(1, 5, 1, 4)});
  for (auto& c : cases) {
    SparseSymbolic s;
    if (!sparse_analyze(c.f, 0, s)) {
      std::printf("%s: analysis refused\n", c.name);
      ++failures;
      continue;
    }
    failures += check(c.f, s, c.name);
  }
  // the 130 x 130 grid: the reference's minimum degree gives nnz(L) = 409164
  {
    const StdForm f = grid(130);
    SparseSymbolic s;
    const auto t0 = std::chrono::steady_clock::now();
    const bool ok = sparse_analyze(f, 0, s);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("grid 130x130: nnz(L)=%lld levels=%d analysis %.3f s\n", s.nnz_l, s.levels(), secs);
    if (!ok || s.nnz_l > 409164 * 13 / 10) ++failures;
  }
  // a fill limit below the true fill refuses the analysis
  {
    SparseSymbolic s;
    if (sparse_analyze(grid(30), 1000, s)) ++failures;
  }
  std::printf("failures %lld\n", failures);
  return failures == 0 ? 0 : 1;
}
