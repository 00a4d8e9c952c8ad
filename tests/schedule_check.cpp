// The GPU work schedule of the sparse L D L' (sparse_schedule, sovereign_b200/csrc/sparse.cpp)
// executed on the CPU exactly as the kernels of sparse_gpu.cu walk it -- per level the pivots,
// the factor's pieces, the combine steps of cut items; the forward and backward solves the same
// way -- on symmetric systems whose graphs hold a dense row (its diagonal collects a term from
// every column and its row of L is long, so items are cut into pieces), positive definite and
// quasi-definite with signed pivots, under every fill-reducing order. The solution must satisfy
// the system to 1e-13 relative (backward error), and the pieces must cover every term once. Prints "failures 0".
#include <cmath>
#include <cstdio>
#include <random>
#include <set>
#include <vector>

#include "sparse.hpp"

using namespace sov;

struct Sys {
  int N;
  std::vector<std::vector<int>> adj;
  std::vector<std::vector<double>> A;  // dense copy (N small enough)
  std::vector<int> sign;               // +1 / -1 expected pivot signs
};

// random SPD-ish block H (n) coupled to m rows: K = [H, B'; B, -delta I] when quasi, else
// [H + B'B-like] as one SPD matrix; node 0 of the first block is joined to every other node (dense)
static Sys make(int n, int m, bool quasi, unsigned seed) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  const int N = n + m;
  Sys S{N, std::vector<std::vector<int>>(N), std::vector<std::vector<double>>(N, std::vector<double>(N, 0.0)),
        std::vector<int>(N, 1)};
  auto link = [&](int a, int b, double v) {
    if (a == b || S.A[a][b] != 0.0) return;
    S.A[a][b] = S.A[b][a] = v;
    S.adj[a].push_back(b);
    S.adj[b].push_back(a);
  };
  for (int j = 0; j + 1 < n; ++j) link(j, j + 1, 0.3 * u(rng));
  for (int j = 1; j < n; ++j) link(0, j, 0.01 * u(rng));  // dense row / column
  for (int i = 0; i < m; ++i) {  // a row over a window of the chain
    const int j0 = static_cast<int>(rng() % (n - 8));
    for (int t = 0; t < 3; ++t) link(n + i, j0 + static_cast<int>(rng() % 8), u(rng));
  }
  for (int k = 0; k < N; ++k) {
    double off = 0.0;
    for (int j = 0; j < N; ++j) off += std::fabs(S.A[k][j]);
    if (k < n || !quasi) S.A[k][k] = off + 1.0;
    else {
      S.A[k][k] = -0.5;  // a moderate delta: the growth of a quasi-definite L D L' is ~ |B|^2 / delta
      S.sign[k] = -1;
    }
  }
  return S;
}

// sparse graph plus a clique of c nodes joined to many others: ordered last, a dense tail
static Sys clique(int n, int c, unsigned seed) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  Sys S{n, std::vector<std::vector<int>>(n), std::vector<std::vector<double>>(n, std::vector<double>(n, 0.0)),
        std::vector<int>(n, 1)};
  auto link = [&](int a, int b, double v) {
    if (a == b || S.A[a][b] != 0.0) return;
    S.A[a][b] = S.A[b][a] = v;
    S.adj[a].push_back(b);
    S.adj[b].push_back(a);
  };
  for (int j = 0; j + 1 < n - c; ++j) link(j, j + 1, 0.3 * u(rng));
  for (int a = n - c; a < n; ++a) {
    for (int b = a + 1; b < n; ++b) link(a, b, 0.05 * u(rng));
    for (int t = 0; t < 12; ++t) link(a, static_cast<int>(rng() % (n - c)), 0.05 * u(rng));
  }
  for (int k = 0; k < n; ++k) {
    double off = 0.0;
    for (int j = 0; j < n; ++j) off += std::fabs(S.A[k][j]);
    S.A[k][k] = off + 1.0;
  }
  return S;
}

// the kernels' walk of the schedule, sequential
static long long run(const Sys& S, SparseOrder order, const char* name, bool use_tail = false, int piece = kSparsePiece,
                     int extra = 0) {
  SparseSymbolic s;
  if (!sparse_analyze_graph(S.adj, 0, s, order)) {
    std::printf("%s: analysis refused\n", name);
    return 1;
  }
  const int m = s.m;
  // the dense trailing block: the full-pattern tail, or more columns (explicit zeros included)
  const int T = use_tail ? std::min(m, sparse_dense_tail(s) + extra) : 0, mt = m - T;
  const SparseSchedule P = sparse_schedule(s, T, piece);
  long long bad = 0;
  // every update term, row entry and column entry is covered exactly once by the pieces
  auto cover = [&](const SparsePieces& pc, size_t total, const char* what) {
    std::vector<int> seen(total, 0);
    for (const auto& p : pc.piece)
      for (int t = p.first; t < p.end; ++t) seen[t]++;
    for (int v : seen)
      if (v != 1) {
        std::printf("%s: %s pieces do not cover every term once\n", name, what);
        ++bad;
        return;
      }
  };
  // per level: the thread-sized pieces (at most kSparseShort terms) first, then the warp pieces
  auto split = [&](const SparsePieces& pc, const char* what) {
    for (int h = 0; h < s.levels(); ++h) {
      const int a = pc.piece_lvl[h], w = pc.warp_lvl[h], e = pc.piece_lvl[h + 1];
      bool ok = a <= w && w <= e;
      for (int q = a; ok && q < w; ++q) ok = pc.piece[q].end - pc.piece[q].first <= kSparseShort && pc.piece[q].slot < 0;
      for (int q = w; ok && q < e; ++q) ok = pc.piece[q].end - pc.piece[q].first > kSparseShort || pc.piece[q].slot >= 0;
      if (!ok) {
        std::printf("%s: %s level %d mixes thread and warp pieces\n", name, what, h);
        ++bad;
        return;
      }
    }
  };
  auto split_levels = [&](const SparsePieces& pc, int levels, const char* what) {
    for (int h = 0; h < levels; ++h) {
      const int a = pc.piece_lvl[h], w = pc.warp_lvl[h], e = pc.piece_lvl[h + 1];
      bool ok = a <= w && w <= e;
      for (int q = a; ok && q < w; ++q) ok = pc.piece[q].end - pc.piece[q].first <= kSparseShort && pc.piece[q].slot < 0;
      for (int q = w; ok && q < e; ++q) ok = pc.piece[q].end - pc.piece[q].first > kSparseShort || pc.piece[q].slot >= 0;
      if (!ok) {
        std::printf("%s: %s level %d mixes thread and warp pieces\n", name, what, h);
        ++bad;
        return;
      }
    }
  };
  split_levels(P.factor, P.levels, "factor");
  split_levels(P.forward, P.levels + (T > 0), "forward");
  split_levels(P.backward, P.levels, "backward");
  cover(P.factor, P.up_col.size(), "factor");
  if (T == 0) {
    cover(P.forward, P.row_pos.size(), "forward");
    cover(P.backward, s.li.size(), "backward");
  }
  // values: [D | L] in elimination order
  std::vector<double> V(m + s.li.size(), 0.0), inv(m), part(std::max(1, std::max(P.factor_slots, P.solve_slots)));
  for (int i = 0; i < m; ++i) {
    V[sparse_slot(s, i, i)] = S.A[i][i];
    for (int j : S.adj[i])
      if (j < i) V[sparse_slot(s, i, j)] = S.A[i][j];
  }
  std::vector<int8_t> sg(m);
  for (int k = 0; k < m; ++k) sg[k] = static_cast<int8_t>(S.sign[s.perm[k]]);
  int drops = 0;
  for (int h = 0; h < P.levels; ++h) {
    for (int q = P.pivot_ptr[h]; q < P.pivot_ptr[h + 1]; ++q) {
      const int k = P.pivot_col[q];
      const double p = V[k];
      const bool drop = !(sg[k] * p > 0.0);
      drops += drop;
      inv[k] = 1.0 / (drop ? sg[k] * 1e128 : p);
    }
    for (int q = P.factor.piece_lvl[h]; q < P.factor.piece_lvl[h + 1]; ++q) {
      const SparsePiece& pc = P.factor.piece[q];
      double acc = 0.0;
      for (int t = pc.first; t < pc.end; ++t) acc += V[m + P.up_a[t]] * V[m + P.up_b[t]] * inv[P.up_col[t]];
      if (pc.slot < 0) V[pc.target] -= acc;
      else part[pc.slot] = acc;
    }
    for (int c = P.factor.comb_lvl[h]; c < P.factor.comb_lvl[h + 1]; ++c) {
      const SparseCombine& cb = P.factor.comb[c];
      double t = 0.0;
      for (int k = 0; k < cb.count; ++k) t += part[cb.first + k];
      V[cb.target] -= t;
    }
  }
  // the block's strict lower triangle, dense (rows and columns relative to mt), from the pattern
  std::vector<double> Ld(static_cast<size_t>(T) * T, 0.0);
  for (int k = mt; k < m; ++k)
    for (int p = s.lp[k]; p < s.lp[k + 1]; ++p) Ld[static_cast<size_t>(s.li[p] - mt) * T + (k - mt)] = V[m + p];
  auto lt = [&](int a, int k) -> double& { return Ld[static_cast<size_t>(a - mt) * T + (k - mt)]; };  // L~_ak
  for (int k = mt; k < m; ++k) {  // the dense tail, column by column
    const double p = V[k];
    const bool drop = !(sg[k] * p > 0.0);
    drops += drop;
    inv[k] = 1.0 / (drop ? sg[k] * 1e128 : p);
    for (int a = k + 1; a < m; ++a)
      for (int b = k + 1; b <= a; ++b) (a == b ? V[a] : lt(a, b)) -= lt(a, k) * lt(b, k) * inv[k];
  }
  if (drops) {
    std::printf("%s: %d pivots with the wrong sign\n", name, drops);
    ++bad;
  }
  // solve K x = b for b = K * ones
  std::vector<double> b(m, 0.0), w(m);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) b[i] += S.A[i][j];
  for (int k = 0; k < m; ++k) w[k] = b[s.perm[k]];
  for (int h = 0; h < P.levels + (T > 0); ++h) {
    for (int q = P.forward.piece_lvl[h]; q < P.forward.piece_lvl[h + 1]; ++q) {
      const SparsePiece& pc = P.forward.piece[q];
      double acc = 0.0;
      for (int t = pc.first; t < pc.end; ++t) acc += V[m + P.row_pos[t]] * inv[P.row_col[t]] * w[P.row_col[t]];
      if (pc.slot < 0) w[pc.target] -= acc;
      else part[pc.slot] = acc;
    }
    for (int c = P.forward.comb_lvl[h]; c < P.forward.comb_lvl[h + 1]; ++c) {
      const SparseCombine& cb = P.forward.comb[c];
      double t = 0.0;
      for (int k = 0; k < cb.count; ++k) t += part[cb.first + k];
      w[cb.target] -= t;
    }
  }
  for (int k = mt; k < m; ++k)  // dense tail: forward, then backward
    for (int i = k + 1; i < m; ++i) w[i] -= lt(i, k) * inv[k] * w[k];
  for (int k = m - 1; k >= mt; --k) {
    double acc = 0.0;
    for (int i = k + 1; i < m; ++i) acc += lt(i, k) * w[i];
    w[k] = (w[k] - acc) * inv[k];
  }
  for (int h = P.levels - 1; h >= 0; --h) {
    for (int q = P.backward.piece_lvl[h]; q < P.backward.piece_lvl[h + 1]; ++q) {
      const SparsePiece& pc = P.backward.piece[q];
      double acc = 0.0;
      for (int p = pc.first; p < pc.end; ++p) acc += V[m + p] * w[s.li[p]];
      if (pc.slot < 0) w[pc.target] = (w[pc.target] - acc) * inv[pc.target];
      else part[pc.slot] = acc;
    }
    for (int c = P.backward.comb_lvl[h]; c < P.backward.comb_lvl[h + 1]; ++c) {
      const SparseCombine& cb = P.backward.comb[c];
      double t = 0.0;
      for (int k = 0; k < cb.count; ++k) t += part[cb.first + k];
      w[cb.target] = (w[cb.target] - t) * inv[cb.target];
    }
  }
  std::vector<double> x(m);
  for (int k = 0; k < m; ++k) x[s.perm[k]] = w[k];
  double err = 0.0, bmax = 0.0;  // backward error: |K x - b|_inf / |b|_inf
  for (int i = 0; i < m; ++i) {
    double r = b[i];
    for (int j = 0; j < m; ++j) r -= S.A[i][j] * x[j];
    err = std::max(err, std::fabs(r));
    bmax = std::max(bmax, std::fabs(b[i]));
  }
  err /= bmax;
  int cut = static_cast<int>(P.factor.comb.size() + P.forward.comb.size() + P.backward.comb.size());
  std::printf("%s [%s, dense tail %d]: N=%d levels=%d pieces %zu/%zu/%zu, cut items %d, |Kx - b| / |b| = %.2e\n", name,
              s.ordering == SparseOrder::kNestedDissection ? "nested dissection" : "minimum degree", T, m, P.levels,
              P.factor.piece.size(), P.forward.piece.size(), P.backward.piece.size(), cut, err);
  if (!(err < 1e-13)) ++bad;
  return bad;
}

int main() {
  long long failures = 0;
  const SparseOrder orders[] = {SparseOrder::kMinimumDegree, SparseOrder::kNestedDissection, SparseOrder::kAuto};
  for (SparseOrder o : orders) {
    failures += run(make(3000, 0, false, 1), o, "definite, dense row, N=3000");
    failures += run(make(2500, 150, true, 2), o, "quasi-definite, dense row, N=2650");
    failures += run(make(40, 10, true, 3), o, "quasi-definite, N=50");
    failures += run(make(3000, 0, false, 1), o, "definite, dense row, N=3000", true);
    failures += run(make(2500, 150, true, 2), o, "quasi-definite, dense row, N=2650", true);
    failures += run(clique(600, 80, 5), o, "definite, 80-node clique, N=600", true);
    failures += run(clique(600, 80, 5), o, "definite, 80-node clique, N=600, 32-term pieces", true, 32);
    failures += run(make(2500, 150, true, 2), o, "quasi-definite, dense row, N=2650, 32-term pieces", true, 32);
    failures += run(clique(600, 80, 5), o, "definite, 80-node clique + 60 sparse columns densely", true, 32, 60);
    failures += run(make(2500, 150, true, 2), o, "quasi-definite, dense row + 300 columns densely", true, 32, 300);
  }
  std::printf("failures %lld\n", failures);
  return failures == 0 ? 0 : 1;
}
