// sparse.cpp -- minimum-degree ordering, symbolic factorization and level schedule (host).
#include "sparse.hpp"

#include <algorithm>
#include <cmath>
#include <set>
#include <thread>
#include <utility>

namespace sov {
namespace {

// Off-diagonal adjacency of A A' (rows sharing a column).
std::vector<std::vector<int>> normal_graph(const StdForm& f) {
  std::vector<std::vector<int>> adj(f.m);
  for (int j = 0; j < f.n; ++j)
    for (int p = f.col_ptr[j]; p < f.col_ptr[j + 1]; ++p)
      for (int q = f.col_ptr[j]; q < f.col_ptr[j + 1]; ++q)
        if (p != q) adj[f.row_idx[p]].push_back(f.row_idx[q]);
  for (auto& l : adj) {
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
  }
  return adj;
}

// Greedy exact minimum degree on the elimination graph (the rule of amd_ordering.cpp:12-130).
bool minimum_degree(std::vector<std::vector<int>> adj, std::size_t fill_limit, std::vector<int>& perm) {
  const int n = static_cast<int>(adj.size());
  perm.assign(n, -1);
  const double dense_degree = std::max(16.0, 10.0 * std::sqrt(static_cast<double>(n)));
  std::vector<char> dense(n, 0);
  std::vector<std::pair<int, int>> dense_nodes;
  for (int i = 0; i < n; ++i)
    if (static_cast<double>(adj[i].size()) > dense_degree) {
      dense[i] = 1;
      dense_nodes.push_back({static_cast<int>(adj[i].size()), i});
    }
  if (!dense_nodes.empty()) {
    for (int i = 0; i < n; ++i) {
      if (dense[i]) {
        std::vector<int>().swap(adj[i]);
        continue;
      }
      auto& l = adj[i];
      l.erase(std::remove_if(l.begin(), l.end(), [&](int w) { return dense[w] != 0; }), l.end());
    }
    std::sort(dense_nodes.begin(), dense_nodes.end());
  }
  const int n_sparse = n - static_cast<int>(dense_nodes.size());
  for (int k = n_sparse; k < n; ++k) perm[k] = dense_nodes[k - n_sparse].second;
  std::set<std::pair<int, int>> queue;
  for (int i = 0; i < n; ++i)
    if (!dense[i]) queue.insert({static_cast<int>(adj[i].size()), i});
  std::size_t nd = dense_nodes.size();
  std::size_t predicted = nd * (nd > 0 ? nd - 1 : 0) / 2;
  std::vector<int> mark(n, -1);
  int stamp = 0;
  for (int k = 0; k < n_sparse; ++k) {
    const int node = queue.begin()->second;
    queue.erase(queue.begin());
    perm[k] = node;
    std::vector<int> clique;
    clique.swap(adj[node]);
    predicted += clique.size();
    if (fill_limit > 0 && predicted > fill_limit) return false;
    for (int v : clique) {
      auto& l = adj[v];
      queue.erase({static_cast<int>(l.size()), v});
      ++stamp;
      std::size_t keep = 0;
      for (int w : l) {
        if (w == node) continue;
        mark[w] = stamp;
        l[keep++] = w;
      }
      l.resize(keep);
      mark[v] = stamp;
      for (int w : clique)
        if (mark[w] != stamp) l.push_back(w);
      queue.insert({static_cast<int>(l.size()), v});
    }
  }
  return true;
}

int position(const SparseSymbolic& s, int col, int row) {
  const auto b = s.li.begin() + s.lp[col], e = s.li.begin() + s.lp[col + 1];
  const auto it = std::lower_bound(b, e, row);
  return (it != e && *it == row) ? static_cast<int>(it - s.li.begin()) : -1;
}

}  // namespace

bool sparse_analyze(const StdForm& f, std::size_t fill_limit, SparseSymbolic& s) {
  const int m = f.m;
  s = SparseSymbolic{};
  s.m = m;
  const auto adj0 = normal_graph(f);
  if (!minimum_degree(adj0, fill_limit, s.perm)) return false;
  s.iperm.assign(m, 0);
  for (int k = 0; k < m; ++k) s.iperm[s.perm[k]] = k;
  // column patterns: col(k) = {i > k adjacent to k} U (col(c) \ {k}) over children c
  std::vector<std::vector<int>> cols(m), children(m);
  s.parent.assign(m, -1);
  std::vector<int> mark(m, -1);
  for (int k = 0; k < m; ++k) {
    std::vector<int>& c = cols[k];
    for (int r : adj0[s.perm[k]]) {
      const int i = s.iperm[r];
      if (i > k && mark[i] != k) {
        mark[i] = k;
        c.push_back(i);
      }
    }
    for (int ch : children[k])
      for (int i : cols[ch])
        if (i > k && mark[i] != k) {
          mark[i] = k;
          c.push_back(i);
        }
    std::sort(c.begin(), c.end());
    if (!c.empty()) {
      s.parent[k] = c.front();
      children[c.front()].push_back(k);
    }
    if (fill_limit > 0 && static_cast<std::size_t>(s.nnz_l) + c.size() > fill_limit) return false;
    s.nnz_l += static_cast<long long>(c.size());
  }
  s.lp.assign(m + 1, 0);
  for (int k = 0; k < m; ++k) s.lp[k + 1] = s.lp[k] + static_cast<int>(cols[k].size());
  s.li.reserve(s.nnz_l);
  for (int k = 0; k < m; ++k) {
    s.li.insert(s.li.end(), cols[k].begin(), cols[k].end());
    const double cc = static_cast<double>(cols[k].size());
    s.flops += cc * cc;
  }
  // the update schedule below holds one entry per rank-1 term: bounded (3.2 GB at the limit)
  if (s.flops > 2.0 * kMaxUpdates) return false;
  // heights and level schedule
  std::vector<int> height(m, 0);
  int hmax = 0;
  for (int k = 0; k < m; ++k) {
    for (int ch : children[k]) height[k] = std::max(height[k], height[ch] + 1);
    hmax = std::max(hmax, height[k]);
  }
  s.lvl_ptr.assign(hmax + 2, 0);
  for (int k = 0; k < m; ++k) s.lvl_ptr[height[k] + 1]++;
  for (int h = 0; h <= hmax; ++h) s.lvl_ptr[h + 1] += s.lvl_ptr[h];
  s.lvl_col.assign(m, 0);
  {
    std::vector<int> fill(s.lvl_ptr.begin(), s.lvl_ptr.end() - 1);
    for (int k = 0; k < m; ++k) s.lvl_col[fill[height[k]]++] = k;
  }
  // rank-1 updates per level, column by column in level order; each column's block of updates is
  // sized up front, so the blocks are filled on several host threads
  std::vector<std::size_t> at(m + 1, 0);
  for (int q = 0; q < m; ++q) {
    const std::size_t nk = static_cast<std::size_t>(s.lp[s.lvl_col[q] + 1] - s.lp[s.lvl_col[q]]);
    at[q + 1] = at[q] + nk * (nk + 1) / 2;
  }
  s.pairs.resize(4 * at[m]);
  s.pair_ptr.assign(hmax + 2, 0);
  for (int h = 0; h <= hmax; ++h) s.pair_ptr[h + 1] = static_cast<int>(at[s.lvl_ptr[h + 1]]);
  auto fill_columns = [&](int q0, int q1) {
    for (int q = q0; q < q1; ++q) {
      const int k = s.lvl_col[q];
      int* out = s.pairs.data() + 4 * at[q];
      for (int a = s.lp[k]; a < s.lp[k + 1]; ++a)
        for (int b = s.lp[k]; b <= a; ++b) {
          const int ia = s.li[a], ib = s.li[b];
          out[0] = k;
          out[1] = a;
          out[2] = b;
          out[3] = ia == ib ? ia : m + position(s, ib, ia);
          out += 4;
        }
    }
  };
  const int nthreads = at[m] > 1000000 ? std::max(1, std::min(16, static_cast<int>(std::thread::hardware_concurrency()))) : 1;
  if (nthreads == 1) {
    fill_columns(0, m);
  } else {
    std::vector<std::thread> pool;
    int q0 = 0;
    for (int t = 0; t < nthreads; ++t) {  // ranges of about equal update counts
      const std::size_t target = at[m] * (t + 1) / nthreads;
      int q1 = static_cast<int>(std::lower_bound(at.begin(), at.end(), target) - at.begin());
      q1 = std::min(m, std::max(q0, q1));
      if (t == nthreads - 1) q1 = m;
      pool.emplace_back(fill_columns, q0, q1);
      q0 = q1;
    }
    for (std::thread& th : pool) th.join();
  }
  // assembly map into [D | L]: A's column j couples rows p >= q with weight a_p a_q
  struct Contrib {
    int t, col;
    double w;
  };
  std::vector<Contrib> cs;
  for (int j = 0; j < f.n; ++j)
    for (int p = f.col_ptr[j]; p < f.col_ptr[j + 1]; ++p)
      for (int q = f.col_ptr[j]; q <= p; ++q) {
        const int i = s.iperm[f.row_idx[p]], k = s.iperm[f.row_idx[q]];
        const int hi = std::max(i, k), lo = std::min(i, k);
        const int t = hi == lo ? hi : m + position(s, lo, hi);
        cs.push_back({t, j, f.val[p] * f.val[q]});
      }
  for (int i = 0; i < m; ++i) cs.push_back({i, -1, 0.0});  // every diagonal gets a target
  std::stable_sort(cs.begin(), cs.end(), [](const Contrib& a, const Contrib& b) { return a.t < b.t; });
  s.asm_ptr.push_back(0);
  for (std::size_t q = 0; q < cs.size(); ++q) {
    if (s.asm_target.empty() || s.asm_target.back() != cs[q].t) {
      if (!s.asm_target.empty()) s.asm_ptr.push_back(static_cast<int>(s.asm_col.size()));
      s.asm_target.push_back(cs[q].t);
    }
    if (cs[q].col >= 0) {
      s.asm_col.push_back(cs[q].col);
      s.asm_w.push_back(cs[q].w);
    }
  }
  s.asm_ptr.push_back(static_cast<int>(s.asm_col.size()));
  return true;
}

}  // namespace sov
