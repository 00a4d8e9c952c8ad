// stdform.cpp -- host-side standard form and normal-matrix assembly maps.
#include "stdform.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <thread>
#include <utility>

namespace sov {
namespace {

void coefficient_range(const double* v, int count, double& lo, double& hi) {
  // interior_point.cpp:46-56 (zeros and non-finite magnitudes are skipped)
  constexpr double kInf = std::numeric_limits<double>::infinity();
  lo = kInf;
  hi = 0.0;
  for (int q = 0; q < count; ++q) {
    const double a = std::abs(v[q]);
    const bool use = a > 0.0 && a < kInf;
    lo = std::min(lo, use ? a : kInf);
    hi = std::max(hi, use ? a : 0.0);
  }
  if (!(lo < kInf)) lo = 0.0;
}

// CSR (row_ptr, col_idx, rval) of an m x n CSC matrix; within a row, columns ascending.
void csr_from_csc(int m, int n, const int* col_ptr, const int* row_idx, const double* val, int* row_ptr,
                  int* col_idx, double* rval, std::vector<int>& fill) {
  std::fill(row_ptr, row_ptr + m + 1, 0);
  for (int p = 0; p < col_ptr[n]; ++p) row_ptr[row_idx[p] + 1]++;
  for (int i = 0; i < m; ++i) row_ptr[i + 1] += row_ptr[i];
  fill.assign(row_ptr, row_ptr + m);
  for (int j = 0; j < n; ++j)
    for (int p = col_ptr[j]; p < col_ptr[j + 1]; ++p) {
      const int q = fill[row_idx[p]]++;
      col_idx[q] = j;
      rval[q] = val[p];
    }
}

// Two passes of row then column scaling by 1/sqrt(max|a|) (interior_point.cpp:370-405), in place.
// Scale factors repeat (many rows / columns share their largest magnitude), so the last value's
// factor is reused: the same arithmetic with fewer square roots and divisions.
void scale_two_pass(int m, int n, const int* col_ptr, const int* row_idx, double* val, double* b, double* c,
                    double* row_scale, double* col_scale, std::vector<double>& rs) {
  double last_in = 1.0, last_out = 1.0;
  auto inv_sqrt = [&](double v) {
    if (v != last_in) {
      last_in = v;
      last_out = 1.0 / std::sqrt(v);
    }
    return last_out;
  };
  const int nnz = col_ptr[n];
  rs.resize(m);
  for (int pass = 0; pass < 2; ++pass) {
    std::fill(rs.begin(), rs.end(), 0.0);
    for (int q = 0; q < nnz; ++q) rs[row_idx[q]] = std::max(rs[row_idx[q]], std::abs(val[q]));
    for (int i = 0; i < m; ++i) {
      rs[i] = rs[i] > 0.0 ? inv_sqrt(rs[i]) : 1.0;
      row_scale[i] *= rs[i];
      b[i] *= rs[i];
    }
    for (int q = 0; q < nnz; ++q) val[q] *= rs[row_idx[q]];
    for (int j = 0; j < n; ++j) {
      double mx = 0.0;
      for (int q = col_ptr[j]; q < col_ptr[j + 1]; ++q) mx = std::max(mx, std::abs(val[q]));
      const double sc = mx > 0.0 ? inv_sqrt(mx) : 1.0;
      for (int q = col_ptr[j]; q < col_ptr[j + 1]; ++q) val[q] *= sc;
      c[j] *= sc;
      col_scale[j] *= sc;
    }
  }
}

void build_csr(StdForm& f) {
  f.row_ptr.resize(f.m + 1);
  f.col_idx.resize(f.nnz());
  f.rval.resize(f.nnz());
  std::vector<int> fill;
  csr_from_csc(f.m, f.n, f.col_ptr.data(), f.row_idx.data(), f.val.data(), f.row_ptr.data(), f.col_idx.data(),
               f.rval.data(), fill);
}

}  // namespace

StdForm build_std_form(const sov_model& p, bool qp, bool enable_scaling) {
  StdForm f;
  f.qp = qp;
  const int ns = p.n, m0 = p.m;
  f.n_struct = ns;
  f.m0 = m0;
  f.shift.assign(ns, 0.0);
  std::vector<uint8_t> free_s(ns, 0);
  std::vector<std::pair<int, double>> ub_cons;
  for (int j = 0; j < ns; ++j) {
    const double lb = p.lb ? p.lb[j] : 0.0;
    const double ub = p.ub ? p.ub[j] : 1e30;
    const bool no_lower = qp && !(lb > -1e29);
    free_s[j] = no_lower ? 1 : 0;
    f.shift[j] = no_lower ? 0.0 : lb;
    if (std::isfinite(ub) && ub < 1e29) {
      const double u = ub - f.shift[j];
      if (!no_lower && u < -1e-12) throw std::runtime_error("Inconsistent bounds for variable x" + std::to_string(j));
      ub_cons.push_back({j, u});
    }
  }
  const int n_ub = static_cast<int>(ub_cons.size());
  const int m = m0 + n_ub;
  int n_slack = n_ub;
  for (int r = 0; r < m0; ++r) n_slack += p.sense[r] != SOV_EQ ? 1 : 0;
  const int n = ns + n_slack;
  f.m = m;
  f.n = n;
  f.b.assign(m, 0.0);
  f.c.assign(n, 0.0);
  f.col_scale.assign(n, 1.0);
  f.row_scale.assign(m, 1.0);
  f.free_col.assign(n, 0);
  std::copy(free_s.begin(), free_s.end(), f.free_col.begin());
  for (int i = 0; i < m0; ++i) f.b[i] = p.rhs[i];

  std::vector<int> ub_row(ns, -1);
  for (int k = 0; k < n_ub; ++k) ub_row[ub_cons[k].first] = m0 + k;

  f.col_ptr.assign(n + 1, 0);
  f.row_idx.reserve(static_cast<std::size_t>(p.col_ptr[ns]) + n_ub + n_slack);
  f.val.reserve(f.row_idx.capacity());
  std::vector<std::pair<int, double>> col;
  for (int j = 0; j < ns; ++j) {
    // fast path: no upper-bound row, rows strictly increasing, no zero or NaN -> copied as is
    if (ub_row[j] < 0) {
      bool plain = true;
      for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k)
        if (!(std::abs(p.values[k]) > 0.0) || (k > p.col_ptr[j] && p.row_idx[k] <= p.row_idx[k - 1])) {
          plain = false;
          break;
        }
      if (plain) {
        for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) {
          if (p.row_idx[k] < m0) f.b[p.row_idx[k]] -= p.values[k] * f.shift[j];
          f.row_idx.push_back(p.row_idx[k]);
          f.val.push_back(p.values[k]);
        }
        f.col_ptr[j + 1] = static_cast<int>(f.row_idx.size());
        continue;
      }
    }
    col.clear();
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) col.push_back({p.row_idx[k], p.values[k]});
    if (ub_row[j] >= 0) col.push_back({ub_row[j], 1.0});
    if (!std::is_sorted(col.begin(), col.end(), [](const auto& a, const auto& b) { return a.first < b.first; }))
      std::sort(col.begin(), col.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    // merge duplicates (a Constraint's name-keyed map sums them), then drop exact zeros
    std::size_t w = 0;
    for (std::size_t q = 0; q < col.size(); ++q) {
      if (w > 0 && col[w - 1].first == col[q].first) col[w - 1].second += col[q].second;
      else col[w++] = col[q];
    }
    col.resize(w);
    for (const auto& e : col) {
      if (e.first < m0) f.b[e.first] -= e.second * f.shift[j];
      if (std::abs(e.second) > 0.0) {
        f.row_idx.push_back(e.first);
        f.val.push_back(e.second);
      }
    }
    f.col_ptr[j + 1] = static_cast<int>(f.row_idx.size());
  }
  for (int k = 0; k < n_ub; ++k) f.b[m0 + k] = ub_cons[k].second;
  int sc = ns;
  for (int r = 0; r < m; ++r) {
    const int kind = r < m0 ? p.sense[r] : SOV_LE;
    if (kind == SOV_EQ) continue;
    f.row_idx.push_back(r);
    f.val.push_back(kind == SOV_LE ? 1.0 : -1.0);
    f.col_ptr[++sc] = static_cast<int>(f.row_idx.size());
  }
  const double sign = p.maximize ? -1.0 : 1.0;
  for (int j = 0; j < ns; ++j) f.c[j] = sign * (p.obj ? p.obj[j] : 0.0);

  if (qp) {
    // build_hessian (qp_interior_point.cpp:68-106)
    std::vector<std::vector<std::pair<int, double>>> qc(n);
    if (p.q_col_ptr) {
      for (int j = 0; j < ns; ++j)
        for (int k = p.q_col_ptr[j]; k < p.q_col_ptr[j + 1]; ++k) {
          const int i = p.q_row_idx[k];
          const double v = sign * p.q_values[k];
          if (i == j) qc[i].push_back({i, v});
          else {
            qc[j].push_back({i, 0.5 * v});
            qc[i].push_back({j, 0.5 * v});
          }
        }
    }
    for (int i = 0; i < ns; ++i) qc[i].push_back({i, 1e-14});
    f.q_ptr.assign(n + 1, 0);
    f.qdiag.assign(n, 0.0);
    for (int j = 0; j < n; ++j) {
      auto& e = qc[j];
      std::stable_sort(e.begin(), e.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      for (std::size_t k = 0; k < e.size();) {
        const int r = e[k].first;
        double v = 0.0;
        for (; k < e.size() && e[k].first == r; ++k) v += e[k].second;
        if (v != 0.0) {
          f.q_idx.push_back(r);
          f.q_val.push_back(v);
          if (r == j) f.qdiag[j] = v;
          else f.q_diagonal = false;
          f.has_quadratic = f.has_quadratic || std::abs(v) > 1e-12;
        }
      }
      f.q_ptr[j + 1] = static_cast<int>(f.q_idx.size());
    }
    // c_eff = sense*c + Q*lb (:206-216) and the gap's objective offset (:2966-2975)
    std::vector<double> qs(n, 0.0);
    for (int j = 0; j < ns; ++j)
      for (int k = f.q_ptr[j]; k < f.q_ptr[j + 1]; ++k) qs[f.q_idx[k]] += f.q_val[k] * f.shift[j];
    double cs = 0.0, sqs = 0.0;
    for (int j = 0; j < ns; ++j) {
      f.c[j] += qs[j];
      cs += f.c[j] * f.shift[j];
      sqs += f.shift[j] * qs[j];
    }
    f.objective_offset = cs - 0.5 * sqs + sign * p.obj_constant;
  }

  coefficient_range(f.val.data(), f.nnz(), f.coef_min_before, f.coef_max_before);
  f.scaling_applied = enable_scaling && m > 0 && n > 0;
  if (f.scaling_applied) {
    std::vector<double> rs;
    scale_two_pass(m, n, f.col_ptr.data(), f.row_idx.data(), f.val.data(), f.b.data(), f.c.data(),
                   f.row_scale.data(), f.col_scale.data(), rs);
  }
  coefficient_range(f.val.data(), f.nnz(), f.coef_min_after, f.coef_max_after);
  build_csr(f);
  return f;
}

bool plain_lp_shape(const sov_model& p, LpShape* s) {
  const int ns = p.n, m0 = p.m;
  int n_ub = 0;
  for (int j = 0; j < ns; ++j) {
    const double ub = p.ub ? p.ub[j] : 1e30;
    if (std::isfinite(ub) && ub < 1e29) ++n_ub;
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k)
      if (!(std::abs(p.values[k]) > 0.0) || (k > p.col_ptr[j] && p.row_idx[k] <= p.row_idx[k - 1])) return false;
  }
  int n_slack = n_ub;
  for (int r = 0; r < m0; ++r) n_slack += p.sense[r] != SOV_EQ ? 1 : 0;
  s->n_struct = ns;
  s->m0 = m0;
  s->n_ub = n_ub;
  s->m = m0 + n_ub;
  s->n = ns + n_slack;
  s->nnz = (p.col_ptr[ns] - p.col_ptr[0]) + n_ub + n_slack;
  return true;
}

void build_plain_lp_into(const sov_model& p, const LpShape& s, bool enable_scaling, const LpFormOut& o,
                         LpFormInfo* info, bool with_rows) {
  // The same arithmetic as build_std_form + scale_two_pass + csr_from_csc, fused into three passes
  // over the entries: (1) copy, with the row counts, the coefficient range and the first row
  // maxima; (2), (3) one scaling pass each, column by column (row scale, column maximum, column
  // scale), the first one also collecting the second pass's row maxima and the second one the
  // final coefficient range and (4) the CSR fill (a pass of its own without scaling). Every value
  // sees the same multiplications in the same order, so the result is bit for bit the general
  // builder's.
  thread_local std::vector<double> rs1, rs2;
  thread_local std::vector<int> fill;
  constexpr double kInf = std::numeric_limits<double>::infinity();
  const int ns = s.n_struct, m0 = s.m0, m = s.m, n = s.n;
  rs1.assign(m, 0.0);
  std::fill(o.row_ptr, o.row_ptr + m + 1, 0);
  double lo = kInf, hi = 0.0;
  auto put = [&](int q, int r, double v) {
    o.row_idx[q] = r;
    o.val[q] = v;
    o.row_ptr[r + 1]++;
    const double a = std::abs(v);
    const bool use = a > 0.0 && a < kInf;
    lo = std::min(lo, use ? a : kInf);
    hi = std::max(hi, use ? a : 0.0);
    rs1[r] = std::max(rs1[r], a);
  };
  for (int i = 0; i < m0; ++i) o.b[i] = p.rhs[i];
  // (1) structural columns: shift by lb, the column's entries, then its upper-bound row
  // (interior_point.cpp:238-247, :289-293); slack (+1) / surplus (-1) columns (:339-350)
  int q = 0, k_ub = 0;
  o.col_ptr[0] = 0;
  for (int j = 0; j < ns; ++j) {
    const double lb = p.lb ? p.lb[j] : 0.0;
    const double ub = p.ub ? p.ub[j] : 1e30;
    o.shift[j] = lb;
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) {
      const int r = p.row_idx[k];
      o.b[r] -= p.values[k] * lb;
      put(q++, r, p.values[k]);
    }
    if (std::isfinite(ub) && ub < 1e29) {
      const double u = ub - lb;
      if (u < -1e-12) throw std::runtime_error("Inconsistent bounds for variable x" + std::to_string(j));
      const int r = m0 + k_ub++;
      o.b[r] = u;
      put(q++, r, 1.0);
    }
    o.col_ptr[j + 1] = q;
  }
  int col = ns;
  for (int r = 0; r < m; ++r) {
    const int kind = r < m0 ? p.sense[r] : SOV_LE;
    if (kind == SOV_EQ) continue;
    put(q++, r, kind == SOV_LE ? 1.0 : -1.0);
    o.col_ptr[++col] = q;
  }
  const double sign = p.maximize ? -1.0 : 1.0;
  for (int j = 0; j < n; ++j) {
    o.c[j] = j < ns ? sign * (p.obj ? p.obj[j] : 0.0) : 0.0;
    o.col_scale[j] = 1.0;
  }
  for (int i = 0; i < m; ++i) o.row_scale[i] = 1.0;
  info->coef_min_before = lo < kInf ? lo : 0.0;
  info->coef_max_before = hi;
  info->scaling_applied = enable_scaling && m > 0 && n > 0;
  // CSR row starts from the counts taken in (1); the entries are filled by the last pass
  for (int i = 0; i < m; ++i) o.row_ptr[i + 1] += o.row_ptr[i];
  fill.assign(o.row_ptr, o.row_ptr + m);
  if (info->scaling_applied) {
    // scale factors 1/sqrt(max|a|): a run of equal maxima (common: many rows and columns share
    // their largest magnitude) reuses the last factor, the same value computed once
    auto inv_sqrt_runs = [](double* v, int len) {
      double last_in = std::numeric_limits<double>::quiet_NaN(), last_out = 1.0;
      for (int k = 0; k < len; ++k) {
        const double x = v[k];
        if (!(x == last_in)) {
          last_in = x;
          last_out = x > 0.0 ? 1.0 / std::sqrt(x) : 1.0;
        }
        v[k] = last_out;
      }
    };
    thread_local std::vector<double> cmx;
    cmx.resize(n);
    rs2.assign(m, 0.0);
    lo = kInf;
    hi = 0.0;
    // (2), (3): rows by 1/sqrt(max|a|), then columns (interior_point.cpp:370-405), twice
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<double>& rs = pass == 0 ? rs1 : rs2;
      inv_sqrt_runs(rs.data(), m);
      for (int i = 0; i < m; ++i) {
        o.row_scale[i] *= rs[i];
        o.b[i] *= rs[i];
      }
      for (int j = 0; j < n; ++j) {
        double mx = 0.0;
        for (int k = o.col_ptr[j]; k < o.col_ptr[j + 1]; ++k) {
          o.val[k] *= rs[o.row_idx[k]];
          mx = std::max(mx, std::abs(o.val[k]));
        }
        cmx[j] = mx;
      }
      inv_sqrt_runs(cmx.data(), n);
      for (int j = 0; j < n; ++j) {
        const double sc = cmx[j];
        for (int k = o.col_ptr[j]; k < o.col_ptr[j + 1]; ++k) {
          o.val[k] *= sc;
          const double a = std::abs(o.val[k]);
          if (pass == 0) {
            rs2[o.row_idx[k]] = std::max(rs2[o.row_idx[k]], a);
          } else {
            const bool use = a > 0.0 && a < kInf;
            lo = std::min(lo, use ? a : kInf);
            hi = std::max(hi, use ? a : 0.0);
            if (with_rows) {
              const int t = fill[o.row_idx[k]]++;  // (4) the CSR entry, in column order per row
              o.col_idx[t] = j;
              o.rval[t] = o.val[k];
            }
          }
        }
        o.c[j] *= sc;
        o.col_scale[j] *= sc;
      }
    }
    info->coef_min_after = lo < kInf ? lo : 0.0;
    info->coef_max_after = hi;
  } else {
    info->coef_min_after = info->coef_min_before;
    info->coef_max_after = info->coef_max_before;
    // (4) CSR
    if (with_rows)
      for (int j = 0; j < n; ++j)
        for (int k = o.col_ptr[j]; k < o.col_ptr[j + 1]; ++k) {
          const int t = fill[o.row_idx[k]]++;
          o.col_idx[t] = j;
          o.rval[t] = o.val[k];
        }
  }
}

namespace {

// Indices 0..n-1 in key order, equal keys in index order: an LSD radix sort (11-bit digits) over
// the key's significant bits, carrying the keys along. Keys are non-negative.
std::vector<uint32_t> stable_key_order(const std::vector<int64_t>& key) {
  const std::size_t n = key.size();
  constexpr int kDigit = 11;
  constexpr std::size_t kBuckets = std::size_t(1) << kDigit;
  std::vector<uint32_t> ia(n), ib(n);
  std::vector<uint64_t> ka(n), kb(n);
  uint64_t mx = 0;
  for (std::size_t i = 0; i < n; ++i) {
    ia[i] = static_cast<uint32_t>(i);
    ka[i] = static_cast<uint64_t>(key[i]);
    mx = std::max(mx, ka[i]);
  }
  int bits = 0;
  while (bits < 64 && (mx >> bits) != 0) ++bits;
  std::vector<std::size_t> cnt(kBuckets);
  for (int sh = 0; sh < bits; sh += kDigit) {
    std::fill(cnt.begin(), cnt.end(), 0);
    for (std::size_t i = 0; i < n; ++i) ++cnt[(ka[i] >> sh) & (kBuckets - 1)];
    std::size_t run = 0;
    for (std::size_t d = 0; d < kBuckets; ++d) {
      const std::size_t c = cnt[d];
      cnt[d] = run;
      run += c;
    }
    for (std::size_t i = 0; i < n; ++i) {
      const std::size_t at = cnt[(ka[i] >> sh) & (kBuckets - 1)]++;
      ib[at] = ia[i];
      kb[at] = ka[i];
    }
    ia.swap(ib);
    ka.swap(kb);
  }
  return ia;
}

template <class Index>
AssemblyMap build_assembly(const StdForm& f, Index index) {
  // contributions (target, column, weight) for every pair p >= q of a column's entries, grouped
  // by target in generation order (column, then entry pair): the gather sums in that order
  std::size_t total = 0;
  for (int j = 0; j < f.n; ++j) {
    const std::size_t k = static_cast<std::size_t>(f.col_ptr[j + 1] - f.col_ptr[j]);
    total += k * (k + 1) / 2;
  }
  std::vector<int64_t> ct;
  std::vector<int> cc;
  std::vector<double> cw;
  ct.reserve(total);
  cc.reserve(total);
  cw.reserve(total);
  for (int j = 0; j < f.n; ++j)
    for (int p = f.col_ptr[j]; p < f.col_ptr[j + 1]; ++p)
      for (int q = f.col_ptr[j]; q <= p; ++q) {
        ct.push_back(index(f.row_idx[p], f.row_idx[q]));
        cc.push_back(j);
        cw.push_back(f.val[p] * f.val[q]);
      }
  const std::vector<uint32_t> order = stable_key_order(ct);
  AssemblyMap am;
  am.ptr.reserve(total + 1);
  am.target.reserve(total);
  am.col.resize(total);
  am.w.resize(total);
  am.ptr.push_back(0);
  for (std::size_t k = 0; k < total; ++k) {
    const uint32_t o = order[k];
    if (am.target.empty() || am.target.back() != ct[o]) {
      if (!am.target.empty()) am.ptr.push_back(static_cast<int>(k));
      am.target.push_back(ct[o]);
    }
    am.col[k] = cc[o];
    am.w[k] = cw[o];
  }
  am.ptr.push_back(static_cast<int>(total));
  if (am.target.empty()) am.ptr.assign(1, 0);
  // every diagonal entry gets a target (rows with no entries still carry the 1e-12 shift)
  am.diag_target.assign(f.m, -1);
  std::vector<int64_t> extra;
  for (int i = 0; i < f.m; ++i) {
    const int64_t t = index(i, i);
    auto it = std::lower_bound(am.target.begin(), am.target.end(), t);
    if (it == am.target.end() || *it != t) extra.push_back(t);
  }
  if (!extra.empty()) {
    // insert empty targets for missing diagonals
    std::vector<int64_t> tg;
    std::vector<int> ptr;
    ptr.push_back(0);
    std::size_t a = 0, e = 0;
    std::vector<int> col;
    std::vector<double> w;
    while (a < am.target.size() || e < extra.size()) {
      if (e < extra.size() && (a >= am.target.size() || extra[e] < am.target[a])) {
        tg.push_back(extra[e++]);
        ptr.push_back(static_cast<int>(col.size()));
      } else {
        tg.push_back(am.target[a]);
        for (int q = am.ptr[a]; q < am.ptr[a + 1]; ++q) {
          col.push_back(am.col[q]);
          w.push_back(am.w[q]);
        }
        ptr.push_back(static_cast<int>(col.size()));
        ++a;
      }
    }
    am.target.swap(tg);
    am.ptr.swap(ptr);
    am.col.swap(col);
    am.w.swap(w);
  }
  for (int i = 0; i < f.m; ++i) {
    const int64_t t = index(i, i);
    am.diag_target[i] = static_cast<int>(std::lower_bound(am.target.begin(), am.target.end(), t) - am.target.begin());
  }
  return am;
}

}  // namespace

// Column-major targets t = c * ld + r (r >= c) come out in order without a global sort: for each
// row c of A (its row-wise copy), the columns j holding it in ascending order, and each entry of j
// at a row r >= c, contribute a_rj a_cj to (r, c). Appending each to a per-row list keeps every
// target's contributions in ascending j, the order the generic builder produces (one entry pair
// per column and target), so the gather sums identically; only the group's distinct rows are sorted.
AssemblyMap build_assembly_dense(const StdForm& f, int ld) {
  // needs strictly increasing rows in every column (as build_std_form leaves them); other input
  // goes through the generic builder
  for (int j = 0; j < f.n; ++j)
    for (int p = f.col_ptr[j] + 1; p < f.col_ptr[j + 1]; ++p)
      if (f.row_idx[p] <= f.row_idx[p - 1])
        return build_assembly(f, [ld](int r, int c) { return static_cast<int64_t>(c) * ld + r; });
  // the row-wise copy, when the form carries none
  std::vector<int> own_ptr, own_idx, fill;
  std::vector<double> own_val;
  const int* row_ptr = f.row_ptr.data();
  const int* col_idx = f.col_idx.data();
  const double* rval = f.rval.data();
  if (static_cast<int>(f.row_ptr.size()) != f.m + 1) {
    own_ptr.resize(f.m + 1);
    own_idx.resize(f.col_ptr[f.n]);
    own_val.resize(f.col_ptr[f.n]);
    csr_from_csc(f.m, f.n, f.col_ptr.data(), f.row_idx.data(), f.val.data(), own_ptr.data(), own_idx.data(),
                 own_val.data(), fill);
    row_ptr = own_ptr.data();
    col_idx = own_idx.data();
    rval = own_val.data();
  }
  std::size_t total = 0;
  for (int j = 0; j < f.n; ++j) {
    const std::size_t k = static_cast<std::size_t>(f.col_ptr[j + 1] - f.col_ptr[j]);
    total += k * (k + 1) / 2;
  }
  // rows c of A in contiguous ranges, one per thread, balanced by the entries each row's columns
  // hold; each range builds its own piece, the pieces are concatenated in row order
  struct Piece {
    std::vector<int64_t> target;
    std::vector<int> end;  // end of each target's contributions within the piece
    std::vector<int> col;
    std::vector<double> w;
    std::vector<std::pair<int, int>> diag;  // (row, target index within the piece)
  };
  auto build_rows = [&](int c0, int c1, Piece& pc) {
    std::vector<int> head(f.m, -1), tail(f.m, -1), rows, next, gcol;
    std::vector<double> gw;
    for (int c = c0; c < c1; ++c) {
      rows.clear();
      next.clear();
      gcol.clear();
      gw.clear();
      for (int pp = row_ptr[c]; pp < row_ptr[c + 1]; ++pp) {
        const int j = col_idx[pp];
        const double vc = rval[pp];
        for (int p = f.col_ptr[j]; p < f.col_ptr[j + 1]; ++p) {
          const int r = f.row_idx[p];
          if (r < c) continue;
          const int k = static_cast<int>(gcol.size());
          gcol.push_back(j);
          gw.push_back(f.val[p] * vc);
          next.push_back(-1);
          if (head[r] < 0) {
            head[r] = k;
            rows.push_back(r);
          } else {
            next[tail[r]] = k;
          }
          tail[r] = k;
        }
      }
      std::sort(rows.begin(), rows.end());
      const int64_t base = static_cast<int64_t>(c) * ld;
      if (rows.empty() || rows.front() != c) {  // every diagonal entry gets a target (the 1e-12 shift)
        pc.diag.push_back({c, static_cast<int>(pc.target.size())});
        pc.target.push_back(base + c);
        pc.end.push_back(static_cast<int>(pc.col.size()));
      }
      for (const int r : rows) {
        if (r == c) pc.diag.push_back({c, static_cast<int>(pc.target.size())});
        pc.target.push_back(base + r);
        for (int k = head[r]; k >= 0; k = next[k]) {
          pc.col.push_back(gcol[k]);
          pc.w.push_back(gw[k]);
        }
        pc.end.push_back(static_cast<int>(pc.col.size()));
        head[r] = -1;
      }
    }
  };
  int nthreads = 1;
  if (total >= 100000) nthreads = static_cast<int>(std::min(8u, std::max(1u, std::thread::hardware_concurrency())));
  std::vector<int> cut(nthreads + 1, f.m);
  cut[0] = 0;
  if (nthreads > 1) {
    std::vector<std::size_t> work(f.m + 1, 0);
    for (int c = 0; c < f.m; ++c) {
      std::size_t wc = 1;
      for (int pp = row_ptr[c]; pp < row_ptr[c + 1]; ++pp) wc += f.col_ptr[col_idx[pp] + 1] - f.col_ptr[col_idx[pp]];
      work[c + 1] = work[c] + wc;
    }
    for (int t = 1; t < nthreads; ++t)
      cut[t] = static_cast<int>(std::lower_bound(work.begin(), work.end(), work[f.m] * t / nthreads) - work.begin());
    for (int t = 1; t <= nthreads; ++t) cut[t] = std::max(cut[t], cut[t - 1]);
  }
  std::vector<Piece> pieces(nthreads);
  if (nthreads == 1) {
    build_rows(0, f.m, pieces[0]);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) pool.emplace_back(build_rows, cut[t], cut[t + 1], std::ref(pieces[t]));
    for (std::thread& th : pool) th.join();
  }
  AssemblyMap am;
  std::size_t ntargets = 0;
  for (const Piece& pc : pieces) ntargets += pc.target.size();
  am.target.reserve(ntargets);
  am.ptr.reserve(ntargets + 1);
  am.col.reserve(total);
  am.w.reserve(total);
  am.ptr.push_back(0);
  am.diag_target.assign(f.m, -1);
  for (const Piece& pc : pieces) {
    const int t0 = static_cast<int>(am.target.size()), k0 = static_cast<int>(am.col.size());
    am.target.insert(am.target.end(), pc.target.begin(), pc.target.end());
    for (const int e : pc.end) am.ptr.push_back(k0 + e);
    am.col.insert(am.col.end(), pc.col.begin(), pc.col.end());
    am.w.insert(am.w.end(), pc.w.begin(), pc.w.end());
    for (const auto& d : pc.diag) am.diag_target[d.first] = t0 + d.second;
  }
  return am;
}

AssemblyMap build_assembly_rowmajor(const StdForm& f, int ld) {
  return build_assembly(f, [ld](int r, int c) { return static_cast<int64_t>(r) * ld + c; });
}

AssemblyMap build_assembly_band(const StdForm& f, int kd) {
  const int64_t m = f.m;
  (void)kd;
  return build_assembly(f, [m](int r, int c) { return static_cast<int64_t>(r - c) * m + c; });
}

XSpace analyze_xspace(const StdForm& f) {
  XSpace xs;
  if (!f.qp || !f.q_diagonal || f.m == 0) return xs;
  for (int j = 0; j < f.n_struct; ++j)
    if (!(f.qdiag[j] > 0.0)) return xs;
  xs.slack_of_row.assign(f.m, -1);
  xs.sigma.assign(f.m, 0.0);
  for (int j = f.n_struct; j < f.n; ++j) {
    if (f.col_ptr[j + 1] - f.col_ptr[j] != 1) return xs;
    const int r = f.row_idx[f.col_ptr[j]];
    xs.slack_of_row[r] = j;
    xs.sigma[r] = f.val[f.col_ptr[j]];
  }
  for (int r = 0; r < f.m; ++r)
    if (xs.slack_of_row[r] < 0) return xs;  // an equality row: stay in y-space
  for (int r = 0; r < f.m; ++r) {
    int lo = f.n_struct, hi = -1;
    for (int p = f.row_ptr[r]; p < f.row_ptr[r + 1]; ++p) {
      const int j = f.col_idx[p];
      if (j >= f.n_struct) continue;
      lo = std::min(lo, j);
      hi = std::max(hi, j);
    }
    if (hi >= lo) xs.kd = std::max(xs.kd, hi - lo);
  }
  xs.eligible = true;
  return xs;
}

namespace {

template <class Index>
AssemblyMap build_xspace_map(const StdForm& f, const XSpace& xs, Index index) {
  struct Contrib {
    int64_t t;
    int col;
    double w;
  };
  std::vector<Contrib> cs;
  for (int r = 0; r < f.m; ++r) {
    const int slack = xs.slack_of_row[r];
    for (int p = f.row_ptr[r]; p < f.row_ptr[r + 1]; ++p) {
      const int jp = f.col_idx[p];
      if (jp >= f.n_struct) continue;
      for (int q = f.row_ptr[r]; q < f.row_ptr[r + 1]; ++q) {
        const int jq = f.col_idx[q];
        if (jq >= f.n_struct || jq > jp) continue;
        cs.push_back({index(jp, jq), slack, f.rval[p] * f.rval[q]});
      }
    }
  }
  for (int j = 0; j < f.n_struct; ++j) cs.push_back({index(j, j), -1, 0.0});  // every diagonal has a target
  std::stable_sort(cs.begin(), cs.end(), [](const Contrib& a, const Contrib& b) { return a.t < b.t; });
  AssemblyMap am;
  am.ptr.push_back(0);
  for (std::size_t k = 0; k < cs.size(); ++k) {
    if (am.target.empty() || am.target.back() != cs[k].t) {
      if (!am.target.empty()) am.ptr.push_back(static_cast<int>(am.col.size()));
      am.target.push_back(cs[k].t);
    }
    if (cs[k].col >= 0) {
      am.col.push_back(cs[k].col);
      am.w.push_back(cs[k].w);
    }
  }
  am.ptr.push_back(static_cast<int>(am.col.size()));
  am.diag_target.assign(f.n_struct, 0);
  for (int j = 0; j < f.n_struct; ++j)
    am.diag_target[j] = static_cast<int>(std::lower_bound(am.target.begin(), am.target.end(), index(j, j)) -
                                         am.target.begin());
  return am;
}

}  // namespace

AssemblyMap build_assembly_xspace(const StdForm& f, const XSpace& xs, int ld) {
  return build_xspace_map(f, xs, [ld](int r, int c) { return static_cast<int64_t>(c) * ld + r; });
}

AssemblyMap build_assembly_xspace_band(const StdForm& f, const XSpace& xs) {
  const int64_t nx = f.n_struct;
  return build_xspace_map(f, xs, [nx](int r, int c) { return static_cast<int64_t>(r - c) * nx + c; });
}

int normal_bandwidth(const StdForm& f) {
  int kd = 0;
  for (int j = 0; j < f.n; ++j) {
    if (f.col_ptr[j + 1] == f.col_ptr[j]) continue;
    kd = std::max(kd, f.row_idx[f.col_ptr[j + 1] - 1] - f.row_idx[f.col_ptr[j]]);
  }
  return kd;
}

}  // namespace sov
