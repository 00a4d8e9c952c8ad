// sparse.cpp -- minimum-degree ordering, symbolic factorization and level schedule (host).
#include "sparse.hpp"

#include <algorithm>
#include <cmath>
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

// Rows of the elimination graph kept in buckets by their current degree bound: O(1) insert and
// remove, and the next pivot is the head of the lowest non-empty bucket.
class DegreeBuckets {
 public:
  explicit DegreeBuckets(int n) : head_(n + 1, -1), next_(n, -1), prev_(n, -1), deg_(n, 0) {}
  void insert(int i, int d) {
    deg_[i] = d;
    prev_[i] = -1;
    next_[i] = head_[d];
    if (head_[d] >= 0) prev_[head_[d]] = i;
    head_[d] = i;
    lowest_ = std::min(lowest_, d);
  }
  void remove(int i) {
    if (prev_[i] >= 0) next_[prev_[i]] = next_[i];
    else head_[deg_[i]] = next_[i];
    if (next_[i] >= 0) prev_[next_[i]] = prev_[i];
  }
  int pop_lowest() {
    while (head_[lowest_] < 0) ++lowest_;
    const int i = head_[lowest_];
    remove(i);
    return i;
  }
  int degree(int i) const { return deg_[i]; }

 private:
  std::vector<int> head_, next_, prev_, deg_;
  int lowest_ = 0;
};

// Approximate minimum degree on the quotient graph (P. R. Amestoy, T. A. Davis, I. S. Duff, "An
// approximate minimum degree ordering algorithm", SIAM J. Matrix Anal. Appl. 17(4), 1996). The
// elimination graph is never formed: an eliminated row becomes an element standing for the clique
// of its uneliminated neighbours, each row keeps the rows it still touches directly plus the
// elements it belongs to, and its degree is the paper's bound
//   |rows adjacent to i| + |L_p \ i| + sum over its other elements e of |L_e \ L_p|,
// so one pivot costs the element lists it touches instead of the square of its clique. Elements
// that fall inside the new one are absorbed. Rows denser than max(16, 10 sqrt(m)) (the paper's
// dense-row cut) are held back and ordered last, sparsest first. Returns false as soon as the
// predicted entries of L pass fill_limit (0 = no limit).
bool minimum_degree(const std::vector<std::vector<int>>& graph, std::size_t fill_limit, std::vector<int>& perm) {
  enum : char { kRow, kElement, kAbsorbed, kHeld };
  const int n = static_cast<int>(graph.size());
  perm.assign(n, -1);
  const double dense_cut = std::max(16.0, 10.0 * std::sqrt(static_cast<double>(n)));
  std::vector<char> state(n, kRow);
  std::vector<std::pair<int, int>> held;  // (degree, row)
  for (int i = 0; i < n; ++i)
    if (static_cast<double>(graph[i].size()) > dense_cut) {
      state[i] = kHeld;
      held.push_back({static_cast<int>(graph[i].size()), i});
    }
  std::sort(held.begin(), held.end());
  const int sparse_rows = n - static_cast<int>(held.size());
  for (std::size_t h = 0; h < held.size(); ++h) perm[sparse_rows + static_cast<int>(h)] = held[h].second;
  std::vector<std::vector<int>> rows(n), elems(n), members(n);
  DegreeBuckets buckets(n);
  for (int i = 0; i < n; ++i) {
    if (state[i] != kRow) continue;
    for (int j : graph[i])
      if (state[j] == kRow) rows[i].push_back(j);
    buckets.insert(i, static_cast<int>(rows[i].size()));
  }
  std::size_t predicted = held.size() * (held.size() > 0 ? held.size() - 1 : 0) / 2;
  std::vector<int> in_lp(n, 0), wtag(n, 0), w(n, 0);
  int remaining = sparse_rows;
  for (int k = 0; k < sparse_rows; ++k) {
    const int p = buckets.pop_lowest();
    const int tag = k + 1;
    perm[k] = p;
    in_lp[p] = tag;
    // L_p: rows adjacent to p directly or through one of its elements, which p absorbs
    std::vector<int> lp;
    for (int j : rows[p])
      if (state[j] == kRow && in_lp[j] != tag) {
        in_lp[j] = tag;
        lp.push_back(j);
      }
    for (int e : elems[p]) {
      if (state[e] != kElement) continue;
      for (int j : members[e])
        if (state[j] == kRow && in_lp[j] != tag) {
          in_lp[j] = tag;
          lp.push_back(j);
        }
      state[e] = kAbsorbed;
      std::vector<int>().swap(members[e]);
    }
    state[p] = kElement;
    std::vector<int>().swap(rows[p]);
    std::vector<int>().swap(elems[p]);
    --remaining;
    predicted += lp.size();
    if (fill_limit > 0 && predicted > fill_limit) return false;
    // every row of L_p: drop absorbed elements and the rows now reached through p, join p
    for (int i : lp) {
      buckets.remove(i);
      auto& E = elems[i];
      E.erase(std::remove_if(E.begin(), E.end(), [&](int e) { return state[e] != kElement; }), E.end());
      auto& R = rows[i];
      R.erase(std::remove_if(R.begin(), R.end(), [&](int j) { return state[j] != kRow || in_lp[j] == tag; }),
              R.end());
    }
    // w[e] = |L_e \ L_p| for the other elements of L_p's rows
    for (int i : lp)
      for (int e : elems[i]) {
        if (wtag[e] != tag) {
          wtag[e] = tag;
          w[e] = static_cast<int>(members[e].size());
        }
        --w[e];
      }
    const int lsize = static_cast<int>(lp.size());
    for (int i : lp) {
      long long d = static_cast<long long>(rows[i].size()) + (lsize - 1);
      for (int e : elems[i]) {
        if (state[e] != kElement) continue;
        if (w[e] == 0) {  // e lies inside L_p: absorbed by p
          state[e] = kAbsorbed;
          std::vector<int>().swap(members[e]);
          continue;
        }
        d += w[e];
      }
      d = std::min<long long>({d, remaining - 1, static_cast<long long>(buckets.degree(i)) + lsize - 1});
      elems[i].push_back(p);
      buckets.insert(i, static_cast<int>(std::max<long long>(d, 0)));
    }
    members[p] = std::move(lp);
  }
  return true;
}

// Nested dissection by level structures (A. George, J. W. H. Liu, "An automatic nested dissection
// algorithm for irregular finite element problems", SIAM J. Numer. Anal. 15(5), 1978): a
// connected part is split by one level of a breadth-first search from a pseudo-peripheral node --
// the smallest level that leaves at least a quarter of the part on each side, cut down to the
// nodes with a neighbour beyond it, or, when smaller, the smallest minimum vertex cover of the
// edges between two adjacent levels over the balanced cuts -- its two sides are ordered first and
// the separator last;
// parts of at most kNdLeaf nodes, or whose search is too shallow to split, take the minimum-degree
// order of their own subgraph. Dense rows (the same cut as minimum_degree) go last. Separators are
// small and the tree is shallow wherever the graph is long and thin, where minimum degree walks
// the graph from its ends and builds an elimination tree as deep as the graph is long.
constexpr int kNdLeaf = 32;

// Minimum vertex cover (Koenig: from a maximum matching) of the bipartite graph of the edges
// between BFS levels k and k + 1 of a part (lv: the nodes of both levels): removing it separates
// levels <= k from levels > k, and it is never larger than either level. loc: scratch, -1
// everywhere, restored.
void cover_separator(const std::vector<std::vector<int>>& graph, const std::vector<int>& part,
                     const std::vector<int>& dist, int id, const int* lv, int nlv, int k, std::vector<int>& loc,
                     std::vector<int>& cover) {
  std::vector<int> U, V;
  for (int t = 0; t < nlv; ++t) {  // the nodes of levels k and k + 1
    const int v = lv[t];
    bool across = false;
    for (int u : graph[v])
      if (part[u] == id && dist[u] == (dist[v] == k ? k + 1 : k)) {
        across = true;
        break;
      }
    if (!across) continue;
    if (dist[v] == k) {
      loc[v] = static_cast<int>(U.size());
      U.push_back(v);
    } else {
      loc[v] = static_cast<int>(V.size());
      V.push_back(v);
    }
  }
  const int nu = static_cast<int>(U.size()), nv = static_cast<int>(V.size());
  std::vector<std::vector<int>> adj(nu);
  for (int a = 0; a < nu; ++a)
    for (int u : graph[U[a]])
      if (part[u] == id && dist[u] == k + 1 && loc[u] >= 0) adj[a].push_back(loc[u]);
  for (int v : U) loc[v] = -1;
  for (int v : V) loc[v] = -1;
  // maximum matching, one breadth-first augmenting search per free vertex of U
  std::vector<int> mate_u(nu, -1), mate_v(nv, -1), prev(nv, -1), seen(nv, -1), queue;
  for (int a0 = 0; a0 < nu; ++a0) {
    queue.assign(1, a0);
    int end_v = -1;
    for (std::size_t h = 0; h < queue.size() && end_v < 0; ++h) {
      const int a = queue[h];
      for (int b : adj[a]) {
        if (seen[b] == a0) continue;
        seen[b] = a0;
        prev[b] = a;
        if (mate_v[b] < 0) {
          end_v = b;
          break;
        }
        queue.push_back(mate_v[b]);
      }
    }
    for (int b = end_v; b >= 0;) {  // flip the path
      const int a = prev[b], next = mate_u[a];
      mate_u[a] = b;
      mate_v[b] = a;
      b = next;
    }
  }
  // Z: reachable from the free vertices of U along alternating paths; cover = (U \ Z) + (V in Z)
  std::vector<char> zu(nu, 0), zv(nv, 0);
  queue.clear();
  for (int a = 0; a < nu; ++a)
    if (mate_u[a] < 0) {
      zu[a] = 1;
      queue.push_back(a);
    }
  for (std::size_t h = 0; h < queue.size(); ++h)
    for (int b : adj[queue[h]]) {
      if (zv[b]) continue;
      zv[b] = 1;
      const int a = mate_v[b];
      if (a >= 0 && !zu[a]) {
        zu[a] = 1;
        queue.push_back(a);
      }
    }
  cover.clear();
  for (int a = 0; a < nu; ++a)
    if (!zu[a]) cover.push_back(U[a]);
  for (int b = 0; b < nv; ++b)
    if (zv[b]) cover.push_back(V[b]);
}

void nested_dissection(const std::vector<std::vector<int>>& graph, std::vector<int>& perm) {
  const int n = static_cast<int>(graph.size());
  perm.assign(n, -1);
  const double dense_cut = std::max(16.0, 10.0 * std::sqrt(static_cast<double>(n)));
  std::vector<int> part(n, 0);  // part id of each node; -1: ordered (separator, leaf or dense)
  std::vector<std::pair<int, int>> held;
  for (int i = 0; i < n; ++i)
    if (static_cast<double>(graph[i].size()) > dense_cut) {
      part[i] = -1;
      held.push_back({static_cast<int>(graph[i].size()), i});
    }
  std::sort(held.begin(), held.end());
  const int sparse_n = n - static_cast<int>(held.size());
  for (std::size_t h = 0; h < held.size(); ++h) perm[sparse_n + static_cast<int>(h)] = held[h].second;
  struct Task {
    std::vector<int> nodes;
    int lo;
  };
  std::vector<Task> stack;
  {
    Task t{{}, 0};
    for (int i = 0; i < n; ++i)
      if (part[i] == 0) t.nodes.push_back(i);
    stack.push_back(std::move(t));
  }
  int next_id = 1;
  std::vector<int> dist(n, -1), loc(n, -1), queue;
  queue.reserve(n);
  // breadth-first search from r inside part id; returns the nodes in visit order, dist set
  auto bfs = [&](int r, int id, std::vector<int>& order) {
    order.clear();
    dist[r] = 0;
    order.push_back(r);
    for (std::size_t h = 0; h < order.size(); ++h) {
      const int u = order[h];
      for (int v : graph[u])
        if (part[v] == id && dist[v] < 0) {
          dist[v] = dist[u] + 1;
          order.push_back(v);
        }
    }
  };
  auto leaf = [&](const std::vector<int>& nodes, int lo) {
    const int k = static_cast<int>(nodes.size());
    for (int q = 0; q < k; ++q) loc[nodes[q]] = q;
    std::vector<std::vector<int>> sub(k);
    for (int q = 0; q < k; ++q)
      for (int v : graph[nodes[q]])
        if (loc[v] >= 0 && part[v] == part[nodes[q]]) sub[q].push_back(loc[v]);
    std::vector<int> sp;
    minimum_degree(sub, 0, sp);
    for (int q = 0; q < k; ++q) perm[lo + q] = nodes[sp[q]];
    for (int v : nodes) {
      loc[v] = -1;
      part[v] = -1;
    }
  };
  std::vector<int> order, order2;
  while (!stack.empty()) {
    Task t = std::move(stack.back());
    stack.pop_back();
    const int id = part[t.nodes[0]];
    // components of the part, each with its own range
    for (int v : t.nodes) dist[v] = -1;
    std::vector<std::vector<int>> comps;
    for (int v : t.nodes)
      if (dist[v] < 0) {
        bfs(v, id, order);
        comps.push_back(order);
      }
    int lo = t.lo;
    for (auto& comp : comps) {
      const int k = static_cast<int>(comp.size());
      const int cid = next_id++;
      for (int v : comp) part[v] = cid;
      if (k <= kNdLeaf) {
        leaf(comp, lo);
        lo += k;
        continue;
      }
      // pseudo-peripheral node: restart from a sparsest node of the last level while the
      // eccentricity grows
      int r = comp[0];
      for (int v : comp)
        if (graph[v].size() < graph[r].size()) r = v;
      for (int v : comp) dist[v] = -1;
      bfs(r, cid, order);
      int ecc = dist[order.back()];
      for (int round = 0; round < 8; ++round) {
        int cand = order.back();
        for (auto it = order.rbegin(); it != order.rend() && dist[*it] == ecc; ++it)
          if (graph[*it].size() < graph[cand].size()) cand = *it;
        for (int v : comp) dist[v] = -1;
        bfs(cand, cid, order2);
        const int ecc2 = dist[order2.back()];
        if (ecc2 <= ecc) {
          for (int v : comp) dist[v] = -1;
          bfs(r, cid, order);  // restore r's levels
          break;
        }
        r = cand;
        ecc = ecc2;
        order.swap(order2);
      }
      if (ecc < 2) {  // too shallow to split
        leaf(comp, lo);
        lo += k;
        continue;
      }
      std::vector<int> width(ecc + 1, 0);
      for (int v : comp) width[dist[v]]++;
      int best = -1, below = 0;
      for (int l = 0; l <= ecc; ++l) {
        const int above = k - below - width[l];
        if (below >= k / 4 && above >= k / 4 && (best < 0 || width[l] < width[best])) best = l;
        below += width[l];
      }
      if (best < 0) {  // no balanced level: the middle one
        below = 0;
        for (int l = 0; l <= ecc; ++l) {
          if (below + width[l] >= k / 2) {
            best = std::max(1, std::min(l, ecc - 1));
            break;
          }
          below += width[l];
        }
      }
      std::vector<int> sideA, sideB, sep;
      for (int v : comp) {
        if (dist[v] < best) {
          sideA.push_back(v);
        } else if (dist[v] > best) {
          sideB.push_back(v);
        } else {
          bool beyond = false;
          for (int u : graph[v])
            if (part[u] == cid && dist[u] == best + 1) {
              beyond = true;
              break;
            }
          (beyond ? sep : sideA).push_back(v);
        }
      }
      // a smaller separator: the smallest minimum vertex cover of the edges between two adjacent
      // levels k, k + 1 among the balanced cuts (at least a quarter of the part on each side);
      // the search order is nondecreasing in distance, so each level is a span of it
      std::vector<int> start(ecc + 2, 0);
      for (int v : order) start[dist[v] + 1]++;
      for (int l = 0; l <= ecc; ++l) start[l + 1] += start[l];
      std::vector<int> cover, best_cover;
      int cut = -1;
      for (int l = 0; l + 1 <= ecc; ++l) {
        const int below_incl = start[l + 1], above_excl = k - start[l + 2];
        if (below_incl < k / 4 || above_excl < k / 4) continue;
        cover_separator(graph, part, dist, cid, order.data() + start[l], start[l + 2] - start[l], l, loc, cover);
        if (cut < 0 || cover.size() < best_cover.size()) {
          best_cover.swap(cover);
          cut = l;
        }
      }
      if (cut >= 0 && best_cover.size() < sep.size()) {
        for (int v : best_cover) dist[v] = -2;  // mark: separator
        sideA.clear();
        sideB.clear();
        for (int v : comp) {
          if (dist[v] == -2) continue;
          (dist[v] <= cut ? sideA : sideB).push_back(v);
        }
        sep.swap(best_cover);
      }
      const int a = static_cast<int>(sideA.size()), b = static_cast<int>(sideB.size());
      for (int q = 0; q < static_cast<int>(sep.size()); ++q) {
        perm[lo + a + b + q] = sep[q];
        part[sep[q]] = -1;
      }
      const int ida = next_id++, idb = next_id++;
      for (int v : sideA) part[v] = ida;
      for (int v : sideB) part[v] = idb;
      if (a) stack.push_back(Task{std::move(sideA), lo});
      if (b) stack.push_back(Task{std::move(sideB), lo + a});
      lo += k;
    }
  }
}

int position(const SparseSymbolic& s, int col, int row) {
  const auto b = s.li.begin() + s.lp[col], e = s.li.begin() + s.lp[col + 1];
  const auto it = std::lower_bound(b, e, row);
  return (it != e && *it == row) ? static_cast<int>(it - s.li.begin()) : -1;
}

}  // namespace

int sparse_slot(const SparseSymbolic& s, int i, int j) {
  const int a = s.iperm[i], b = s.iperm[j];
  if (a == b) return a;
  const int lo = std::min(a, b), hi = std::max(a, b);
  const int p = position(s, lo, hi);
  return p < 0 ? -1 : s.m + p;
}

bool sparse_analyze(const StdForm& f, std::size_t fill_limit, SparseSymbolic& s, SparseOrder order) {
  if (!sparse_analyze_graph(normal_graph(f), fill_limit, s, order)) return false;
  const int m = f.m;
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

namespace {

// Column patterns of L in the order perm: col(k) = {i > k adjacent to k} U (col(c) \ {k}) over the
// children c of k; the elimination tree and each column's height in it. False when the entries of
// L pass fill_limit (0 = no limit).
struct Patterns {
  std::vector<int> perm, iperm, parent, height;
  std::vector<std::vector<int>> cols;
  long long nnz_l = 0;
  double flops = 0.0;
  int hmax = 0;
};

bool column_patterns(const std::vector<std::vector<int>>& adj, std::vector<int> perm, std::size_t fill_limit,
                     Patterns& P) {
  const int m = static_cast<int>(adj.size());
  P = Patterns{};
  P.perm = std::move(perm);
  P.iperm.assign(m, 0);
  for (int k = 0; k < m; ++k) P.iperm[P.perm[k]] = k;
  P.cols.assign(m, {});
  std::vector<std::vector<int>> children(m);
  P.parent.assign(m, -1);
  P.height.assign(m, 0);
  std::vector<int> mark(m, -1);
  for (int k = 0; k < m; ++k) {
    std::vector<int>& c = P.cols[k];
    for (int r : adj[P.perm[k]]) {
      const int i = P.iperm[r];
      if (i > k && mark[i] != k) {
        mark[i] = k;
        c.push_back(i);
      }
    }
    for (int ch : children[k]) {
      for (int i : P.cols[ch])
        if (i > k && mark[i] != k) {
          mark[i] = k;
          c.push_back(i);
        }
      P.height[k] = std::max(P.height[k], P.height[ch] + 1);
    }
    P.hmax = std::max(P.hmax, P.height[k]);
    std::sort(c.begin(), c.end());
    if (!c.empty()) {
      P.parent[k] = c.front();
      children[c.front()].push_back(k);
    }
    P.nnz_l += static_cast<long long>(c.size());
    if (fill_limit > 0 && static_cast<std::size_t>(P.nnz_l) > fill_limit) return false;
    const double cc = static_cast<double>(c.size());
    P.flops += cc * cc;
  }
  return true;
}

// Estimated GPU time of one factorization: every level costs its grid barriers, every rank-1
// term its loads.
double factor_cost(const Patterns& P) { return (P.hmax + 1) * 5e-6 + P.flops * 1e-11; }

}  // namespace

bool sparse_analyze_graph(const std::vector<std::vector<int>>& adj0, std::size_t fill_limit, SparseSymbolic& s,
                          SparseOrder order) {
  const int m = static_cast<int>(adj0.size());
  s = SparseSymbolic{};
  s.m = m;
  Patterns P, Q;
  bool have = false;
  if (order != SparseOrder::kNestedDissection) {
    std::vector<int> perm;
    have = minimum_degree(adj0, fill_limit, perm) && column_patterns(adj0, std::move(perm), fill_limit, P);
    s.ordering = SparseOrder::kMinimumDegree;
  }
  // nested dissection when asked for, or when the minimum-degree tree is deep enough for its
  // barriers to dominate and the dissection order costs less
  if (order == SparseOrder::kNestedDissection || (order == SparseOrder::kAuto && (!have || P.hmax >= 64))) {
    std::vector<int> perm;
    nested_dissection(adj0, perm);
    const bool ok = column_patterns(adj0, std::move(perm), fill_limit, Q);
    if (ok && (order == SparseOrder::kNestedDissection || !have || factor_cost(Q) < 0.8 * factor_cost(P))) {
      P = std::move(Q);
      have = true;
      s.ordering = SparseOrder::kNestedDissection;
    } else if (order == SparseOrder::kNestedDissection) {
      return false;
    }
  }
  if (!have) return false;
  s.perm = std::move(P.perm);
  s.iperm = std::move(P.iperm);
  s.parent = std::move(P.parent);
  s.nnz_l = P.nnz_l;
  s.flops = P.flops;
  std::vector<std::vector<int>>& cols = P.cols;
  const std::vector<int>& height = P.height;
  const int hmax = P.hmax;
  s.lp.assign(m + 1, 0);
  for (int k = 0; k < m; ++k) s.lp[k + 1] = s.lp[k] + static_cast<int>(cols[k].size());
  s.li.reserve(s.nnz_l);
  for (int k = 0; k < m; ++k) s.li.insert(s.li.end(), cols[k].begin(), cols[k].end());
  // the update schedule below holds one entry per rank-1 term: bounded (3.2 GB at the limit)
  if (s.flops > 2.0 * kMaxUpdates) return false;
  // level schedule
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
  return true;
}

namespace {

void add_item(SparsePieces& P, int first, int end, int target, int* slots, bool keep_empty, int piece = kSparsePiece) {
  const int len = end - first;
  if (len == 0 && !keep_empty) return;
  if (len <= kSparseShort) {
    P.piece.push_back({first, end, target, -1});
    return;
  }
  if (len <= piece) {
    P.pending_long.push_back({first, end, target, -1});
    return;
  }
  const int n = (len + piece - 1) / piece;
  P.comb.push_back({target, *slots, n, 0});
  for (int q = 0; q < n; ++q)
    P.pending_long.push_back({first + q * piece, std::min(end, first + (q + 1) * piece), target, *slots + q});
  *slots += n;
}

void close_level(SparsePieces& P) {
  P.warp_lvl.push_back(static_cast<int>(P.piece.size()));
  P.piece.insert(P.piece.end(), P.pending_long.begin(), P.pending_long.end());
  P.pending_long.clear();
  P.piece_lvl.push_back(static_cast<int>(P.piece.size()));
  P.comb_lvl.push_back(static_cast<int>(P.comb.size()));
}

}  // namespace

SparsePieces row_pieces(const std::vector<int>& ptr, int* slots) {
  SparsePieces P;
  *slots = 0;
  for (std::size_t i = 0; i + 1 < ptr.size(); ++i) add_item(P, ptr[i], ptr[i + 1], static_cast<int>(i), slots, false);
  close_level(P);
  return P;
}

int sparse_dense_tail(const SparseSymbolic& s) {
  int t = 0;
  for (int k = s.m - 1; k >= 0 && s.lp[k + 1] - s.lp[k] == s.m - 1 - k; --k) ++t;
  return t;
}

int sparse_dense_block(const SparseSymbolic& s, double sparse_cost, int min_block) {
  const int m = s.m, full = sparse_dense_tail(s);
  // terms of the columns before k: prefix sums of colcount (colcount + 1) / 2
  std::vector<double> before(m + 1, 0.0);
  for (int k = 0; k < m; ++k) {
    const double c = s.lp[k + 1] - s.lp[k];
    before[k + 1] = before[k] + 0.5 * c * (c + 1.0);
  }
  int best = 0;
  double best_cost = sparse_cost * before[m];
  for (int T = std::max(full, 1); T <= m; T += (T < full + 16 ? 1 : 16)) {
    const double cost = sparse_cost * before[m - T] + static_cast<double>(T) * T * T / 6.0;
    if (cost < best_cost) {
      best_cost = cost;
      best = T;
    }
  }
  return best >= min_block ? best : 0;
}

SparseSchedule sparse_schedule(const SparseSymbolic& s, int tail, int piece) {
  SparseSchedule S;
  const int m = s.m, levels = s.levels(), mt = m - tail;
  S.tail = tail;
  // level of each column; the levels that hold a column before the tail
  std::vector<int> level(m, 0);
  for (int h = 0; h < levels; ++h)
    for (int c = s.lvl_ptr[h]; c < s.lvl_ptr[h + 1]; ++c) level[s.lvl_col[c]] = h;
  int hn = 0;
  for (int k = 0; k < mt; ++k) hn = std::max(hn, level[k] + 1);
  if (tail == 0) hn = levels;
  S.levels = hn;
  S.pivot_ptr.assign(1, 0);
  for (int h = 0; h < hn; ++h) {
    for (int c = s.lvl_ptr[h]; c < s.lvl_ptr[h + 1]; ++c)
      if (s.lvl_col[c] < mt) S.pivot_col.push_back(s.lvl_col[c]);
    S.pivot_ptr.push_back(static_cast<int>(S.pivot_col.size()));
  }
  // updates grouped by (level, destination), schedule order kept within a group: two stable
  // counting sorts (by destination, then by level), linear in the number of updates; a tail
  // column's own updates are left to the dense factorization
  const size_t n_all = s.pairs.size() / 4;
  const int n_dst = m + static_cast<int>(s.li.size());
  std::vector<int> level_of(n_all);
  for (int h = 0; h < levels; ++h)
    for (int u = s.pair_ptr[h]; u < s.pair_ptr[h + 1]; ++u) level_of[u] = h;
  std::vector<int> keep;
  keep.reserve(n_all);
  for (size_t u = 0; u < n_all; ++u)
    if (s.pairs[4 * u] < mt) keep.push_back(static_cast<int>(u));
  const size_t n_up = keep.size();
  std::vector<int> by_dst(n_up), order(n_up);
  {
    std::vector<size_t> cnt(n_dst + 1, 0);
    for (int u : keep) cnt[s.pairs[4 * u + 3] + 1]++;
    for (int d = 0; d < n_dst; ++d) cnt[d + 1] += cnt[d];
    for (int u : keep) by_dst[cnt[s.pairs[4 * u + 3]]++] = u;
    std::vector<size_t> lc(levels + 1, 0);
    for (int u : keep) lc[level_of[u] + 1]++;
    for (int h = 0; h < levels; ++h) lc[h + 1] += lc[h];
    for (size_t q = 0; q < n_up; ++q) {
      const int u = by_dst[q];
      order[lc[level_of[u]]++] = u;
    }
  }
  S.up_col.resize(n_up);
  S.up_a.resize(n_up);
  S.up_b.resize(n_up);
  for (size_t q = 0; q < n_up; ++q) {
    const int u = order[q];
    S.up_col[q] = s.pairs[4 * u];
    S.up_a[q] = s.pairs[4 * u + 1];
    S.up_b[q] = s.pairs[4 * u + 2];
  }
  size_t q = 0;
  for (int h = 0; h < hn; ++h) {
    while (q < n_up && level_of[order[q]] == h) {
      const int dst = s.pairs[4 * order[q] + 3];
      size_t e = q + 1;
      while (e < n_up && level_of[order[e]] == h && s.pairs[4 * order[e] + 3] == dst) ++e;
      add_item(S.factor, static_cast<int>(q), static_cast<int>(e), dst, &S.factor_slots, false, piece);
      q = e;
    }
    close_level(S.factor);
  }
  // rows of L for the forward solve (each row's entries in column order)
  std::vector<int> row_ptr(m + 1, 0);
  S.row_pos.resize(s.li.size());
  S.row_col.resize(s.li.size());
  for (int i : s.li) row_ptr[i + 1]++;
  for (int i = 0; i < m; ++i) row_ptr[i + 1] += row_ptr[i];
  {
    std::vector<int> fill(row_ptr.begin(), row_ptr.end() - 1);
    for (int k = 0; k < m; ++k)
      for (int p = s.lp[k]; p < s.lp[k + 1]; ++p) {
        const int t = fill[s.li[p]]++;
        S.row_pos[t] = p;
        S.row_col[t] = k;
      }
  }
  for (int h = 0; h < hn; ++h) {
    for (int c = s.lvl_ptr[h]; c < s.lvl_ptr[h + 1]; ++c) {
      const int k = s.lvl_col[c];
      if (k < mt) add_item(S.forward, row_ptr[k], row_ptr[k + 1], k, &S.solve_slots, false, piece);
    }
    close_level(S.forward);
  }
  if (tail > 0) {  // the tail rows' sums over the columns before the tail, in one more level
    for (int k = mt; k < m; ++k) {
      int e = row_ptr[k];
      while (e < row_ptr[k + 1] && S.row_col[e] < mt) ++e;
      add_item(S.forward, row_ptr[k], e, k, &S.solve_slots, false, piece);
    }
    close_level(S.forward);
  }
  for (int h = 0; h < hn; ++h) {  // every column, empty ones too (x_k = y_k / D_k)
    for (int c = s.lvl_ptr[h]; c < s.lvl_ptr[h + 1]; ++c) {
      const int k = s.lvl_col[c];
      if (k < mt) add_item(S.backward, s.lp[k], s.lp[k + 1], k, &S.solve_slots, true, piece);
    }
    close_level(S.backward);
  }
  return S;
}

}  // namespace sov
