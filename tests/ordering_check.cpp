// The host ordering and symbolic analysis of the sparse L D L' (sovereign_b200/csrc/sparse.cpp),
// without a GPU: on grid-network and random normal-matrix patterns, and on the KKT pattern of a
// QP with a tridiagonal Hessian, every order (minimum degree, nested dissection, automatic) must
// be a permutation, the column patterns of L must equal a brute-force symbolic elimination in that
// order, the elimination tree must be the first off-diagonal row of each column, the level
// schedule must cover every column once with children below their parents and every update must
// land on an entry of L; the minimum-degree fill on the 130 x 130 grid must stay near the
// reference's nnz(L) = 409164, and on the long, thin KKT pattern nested dissection must cut the
// elimination tree's height from thousands of levels to a few hundred. Prints "failures 0".
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

// brute force: eliminate in the given order on an explicit adjacency matrix (original indices)
static long long check_graph(const std::vector<std::vector<int>>& adj, const SparseSymbolic& s, const char* name) {
  const int m = static_cast<int>(adj.size());
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
  for (int i = 0; i < m; ++i)
    for (int j : adj[i]) g[s.iperm[i]].insert(s.iperm[j]);
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
  // every update term: its destination is a diagonal or an entry of L
  for (std::size_t u = 0; u < s.pairs.size() / 4; ++u) {
    const int dst = s.pairs[4 * u + 3];
    if (dst < 0 || dst >= m + static_cast<int>(s.li.size())) ++bad;
  }
  // every edge of the graph has a value slot
  for (int i = 0; i < m; ++i)
    for (int j : adj[i])
      if (sparse_slot(s, i, j) < m) ++bad;
  const char* order = s.ordering == SparseOrder::kNestedDissection ? "nested dissection" : "minimum degree";
  std::printf("%s [%s]: m=%d nnz(L)=%lld levels=%d mismatches=%lld\n", name, order, m, s.nnz_l, s.levels(), bad);
  return bad;
}

// off-diagonal adjacency of A A'
static std::vector<std::vector<int>> normal_adjacency(const StdForm& f) {
  std::vector<std::set<int>> g(f.m);
  for (int j = 0; j < f.n; ++j)
    for (int p = f.col_ptr[j]; p < f.col_ptr[j + 1]; ++p)
      for (int q = f.col_ptr[j]; q < f.col_ptr[j + 1]; ++q)
        if (p != q) g[f.row_idx[p]].insert(f.row_idx[q]);
  std::vector<std::vector<int>> adj(f.m);
  for (int i = 0; i < f.m; ++i) adj[i].assign(g[i].begin(), g[i].end());
  return adj;
}

// KKT pattern of min sum w/2 (x_{j+1} - x_j)^2 + ... over 0 <= x <= 2 with a covering row per block
// of 8 columns and one budget row: IPM columns x, block surpluses, upper-bound slacks; rows block,
// budget, upper bounds (the coupled_chain_qp shape)
static std::vector<std::vector<int>> chain_kkt(int n) {
  const int block = 8, nb = (n + block - 1) / block;
  const int ncol = n + nb + n, N = ncol + nb + 1 + n;
  std::vector<std::set<int>> g(N);
  auto edge = [&](int a, int b) {
    g[a].insert(b);
    g[b].insert(a);
  };
  for (int j = 0; j + 1 < n; ++j) edge(j, j + 1);
  for (int j = 0; j < n; ++j) {
    edge(j, ncol + j / block);
    edge(j, ncol + nb);
    edge(j, ncol + nb + 1 + j);
    edge(n + nb + j, ncol + nb + 1 + j);
  }
  for (int k = 0; k < nb; ++k) edge(n + k, ncol + k);
  std::vector<std::vector<int>> adj(N);
  for (int i = 0; i < N; ++i) adj[i].assign(g[i].begin(), g[i].end());
  return adj;
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
  const SparseOrder orders[] = {SparseOrder::kMinimumDegree, SparseOrder::kNestedDissection, SparseOrder::kAuto};
  for (auto& c : cases) {
    for (SparseOrder o : orders) {
      SparseSymbolic s;
      if (!sparse_analyze(c.f, 0, s, o)) {
        std::printf("%s: analysis refused\n", c.name);
        ++failures;
        continue;
      }
      failures += check_graph(normal_adjacency(c.f), s, c.name);
    }
  }
  // the KKT pattern of a QP whose Hessian couples neighbours
  {
    const auto adj = chain_kkt(1000);
    SparseSymbolic md, nd, au;
    const bool ok = sparse_analyze_graph(adj, 0, md, SparseOrder::kMinimumDegree) &&
                    sparse_analyze_graph(adj, 0, nd, SparseOrder::kNestedDissection) &&
                    sparse_analyze_graph(adj, 0, au, SparseOrder::kAuto);
    if (!ok) {
      std::printf("chain KKT: analysis refused\n");
      ++failures;
    } else {
      failures += check_graph(adj, md, "chain KKT n=1000");
      failures += check_graph(adj, nd, "chain KKT n=1000");
      failures += check_graph(adj, au, "chain KKT n=1000");
      if (md.levels() < 1000 || nd.levels() > 200 || au.ordering != SparseOrder::kNestedDissection) {
        std::printf("chain KKT: minimum degree %d levels, nested dissection %d levels\n", md.levels(), nd.levels());
        ++failures;
      }
    }
  }
  // the 130 x 130 grid: the reference's minimum degree gives nnz(L) = 409164
  {
    const StdForm f = grid(130);
    SparseSymbolic s, a;
    const auto t0 = std::chrono::steady_clock::now();
    const bool ok = sparse_analyze(f, 0, s, SparseOrder::kMinimumDegree);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("grid 130x130 [minimum degree]: nnz(L)=%lld levels=%d analysis %.3f s\n", s.nnz_l, s.levels(), secs);
    if (!ok || s.nnz_l > 409164 * 13 / 10) ++failures;
    // the automatic choice never takes more levels and more fill at once
    const bool ok2 = sparse_analyze(f, 0, a, SparseOrder::kAuto);
    std::printf("grid 130x130 [automatic]: nnz(L)=%lld levels=%d\n", a.nnz_l, a.levels());
    if (!ok2 || (a.levels() > s.levels() && a.nnz_l > s.nnz_l)) ++failures;
  }
  // a fill limit below the true fill refuses the analysis
  {
    SparseSymbolic s;
    for (SparseOrder o : orders)
      if (sparse_analyze(grid(30), 1000, s, o)) ++failures;
  }
  std::printf("failures %lld\n", failures);
  return failures == 0 ? 0 : 1;
}
