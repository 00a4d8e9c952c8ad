// presolve.cpp -- LP presolve and postsolve in index form, around the GPU engine.
//
// The reference presolves every LP before its solvers (solver/core/src/engine.cpp:108-176,
// solver/presolve/src/presolve.cpp) and maps the answer back; a caller of this library that skips
// the reference's engine gets the same service here, on the column-compressed model, with the
// row multipliers recovered as well (the reference's recovery drops them). Reductions, repeated
// until a pass changes nothing (at most 20 passes):
//   * fixed columns (lb = ub): the value moves into the right-hand sides and the objective constant;
//   * empty rows: checked against their sense and dropped (else the model is infeasible);
//   * singleton rows a x_j (<=, >=, =) b: turned into a bound on x_j (an equality fixes it);
//   * empty columns: set to the bound their cost prefers (no such bound: unbounded).
// Postsolve: kept columns and rows take the reduced answer; removed columns their fixed values;
// removed singleton rows, in reverse order of removal, the multiplier y_i = d_j / a_ij that moves
// the reduced cost d_j of their column onto the row when the row's bound is the one x_j sits on
// (and the sign fits the row's sense), else 0; empty rows 0. Reduced costs of removed columns are
// c_j - sum_i a_ij y_i. The objective is evaluated on the original model.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "errors.hpp"
#include "sov_ipm.h"

struct sov_presolve {
  // the original model (borrowed) and the reduced one (owned)
  const sov_model* orig = nullptr;
  std::vector<int32_t> col_ptr, row_idx;
  std::vector<double> values, obj, lb, ub, rhs;
  std::vector<int8_t> sense;
  sov_model reduced{};
  std::vector<int32_t> col_map, row_map;  // reduced -> original
  std::vector<double> fixed;              // original column -> value once removed (NaN: kept)
  std::vector<char> row_kept;
  struct Removed {
    int row, col;  // singleton row and its column (col -1: an empty row)
    double a;
  };
  std::vector<Removed> removed_rows;  // in order of removal
  int status = -1;                    // -1 reduced model to solve; else a decided status
  std::string message;
  int rows_removed = 0, cols_removed = 0, bounds_tightened = 0, passes = 0;
};

namespace {

constexpr double kTol = 1e-9;
const double kNaN = std::numeric_limits<double>::quiet_NaN();

bool finite_lb(double v) { return v > -1e29; }
bool finite_ub(double v) { return v < 1e29; }

void run(sov_presolve& P) {
  const sov_model& p = *P.orig;
  const int n = p.n, m = p.m;
  const double sign = p.maximize ? -1.0 : 1.0;
  std::vector<double> lb(n), ub(n), rhs(p.rhs, p.rhs + m);
  for (int j = 0; j < n; ++j) {
    lb[j] = p.lb ? p.lb[j] : 0.0;
    ub[j] = p.ub ? p.ub[j] : 1e30;
  }
  // rows by their entries (CSR) for the singleton scan; active counts
  std::vector<int> rp(m + 1, 0), rc(p.col_ptr[n]);
  std::vector<double> rv(p.col_ptr[n]);
  for (int k = 0; k < p.col_ptr[n]; ++k) rp[p.row_idx[k] + 1]++;
  for (int i = 0; i < m; ++i) rp[i + 1] += rp[i];
  {
    std::vector<int> at(rp.begin(), rp.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) {
        rc[at[p.row_idx[k]]] = j;
        rv[at[p.row_idx[k]]++] = p.values[k];
      }
  }
  std::vector<char> col_on(n, 1), row_on(m, 1);
  std::vector<int> row_cnt(m), col_cnt(n);
  for (int i = 0; i < m; ++i) row_cnt[i] = rp[i + 1] - rp[i];
  for (int j = 0; j < n; ++j) col_cnt[j] = p.col_ptr[j + 1] - p.col_ptr[j];
  P.fixed.assign(n, kNaN);
  double constant = p.obj_constant;
  auto fail = [&](int status, const std::string& why) {
    P.status = status;
    P.message = why;
  };
  auto fix = [&](int j, double v) {
    col_on[j] = 0;
    P.fixed[j] = v;
    ++P.cols_removed;
    constant += (p.obj ? p.obj[j] : 0.0) * v;
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) {
      const int i = p.row_idx[k];
      if (!row_on[i]) continue;
      rhs[i] -= p.values[k] * v;
      --row_cnt[i];
    }
  };
  bool changed = true;
  while (changed && P.passes < 20 && P.status < 0) {
    changed = false;
    ++P.passes;
    // fixed columns
    for (int j = 0; j < n && P.status < 0; ++j) {
      if (!col_on[j] || !finite_ub(ub[j]) || !finite_lb(lb[j])) continue;
      const double scale = 1.0 + std::max(std::fabs(lb[j]), std::fabs(ub[j]));
      if (lb[j] > ub[j] + kTol * scale) {
        fail(SOV_INFEASIBLE, "Infeasible (presolve): bounds of x" + std::to_string(j) + " cross");
      } else if (ub[j] - lb[j] <= kTol * scale) {
        fix(j, lb[j] == ub[j] ? lb[j] : 0.5 * (lb[j] + ub[j]));
        changed = true;
      }
    }
    // empty and singleton rows
    for (int i = 0; i < m && P.status < 0; ++i) {
      if (!row_on[i] || row_cnt[i] > 1) continue;
      const int s = p.sense[i];
      if (row_cnt[i] == 0) {
        const double b = rhs[i], tol = kTol * (1.0 + std::fabs(p.rhs[i]));
        const bool ok = s == SOV_LE ? 0.0 <= b + tol : s == SOV_GE ? 0.0 >= b - tol : std::fabs(b) <= tol;
        if (!ok) {
          fail(SOV_INFEASIBLE, "Infeasible (presolve): empty row " + std::to_string(i) + " cannot hold");
          break;
        }
        row_on[i] = 0;
        P.removed_rows.push_back({i, -1, 0.0});
        ++P.rows_removed;
        changed = true;
        continue;
      }
      int j = -1;
      double a = 0.0;
      for (int e = rp[i]; e < rp[i + 1]; ++e)
        if (col_on[rc[e]]) {
          j = rc[e];
          a = rv[e];
        }
      if (j < 0 || a == 0.0) continue;  // an explicit zero: leave the row to the solver
      const double v = rhs[i] / a;
      const bool upper = (s == SOV_LE) == (a > 0.0);  // a x <= b with a > 0, or >= with a < 0
      if (s == SOV_EQ) {
        lb[j] = std::max(lb[j], v);
        ub[j] = std::min(ub[j], v);
        if (lb[j] > ub[j] + kTol * (1.0 + std::fabs(v))) {
          fail(SOV_INFEASIBLE, "Infeasible (presolve): row " + std::to_string(i) + " fixes x" + std::to_string(j) +
                                   " outside its bounds");
          break;
        }
        lb[j] = ub[j] = v;
      } else if (upper) {
        if (v < ub[j]) ub[j] = v;
      } else {
        if (v > lb[j]) lb[j] = v;
      }
      ++P.bounds_tightened;
      row_on[i] = 0;
      for (int e = rp[i]; e < rp[i + 1]; ++e)
        if (col_on[rc[e]]) --col_cnt[rc[e]];
      P.removed_rows.push_back({i, j, a});
      ++P.rows_removed;
      changed = true;
    }
    // empty columns
    for (int j = 0; j < n && P.status < 0; ++j) {
      if (!col_on[j]) continue;
      int live = 0;
      for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) live += row_on[p.row_idx[k]] ? 1 : 0;
      if (live > 0) continue;
      const double c = sign * (p.obj ? p.obj[j] : 0.0);
      double v;
      if (c > 0.0) {
        if (!finite_lb(lb[j])) {
          fail(SOV_UNBOUNDED, "Unbounded (presolve): x" + std::to_string(j) + " is in no row and its cost falls");
          break;
        }
        v = lb[j];
      } else if (c < 0.0) {
        if (!finite_ub(ub[j])) {
          fail(SOV_UNBOUNDED, "Unbounded (presolve): x" + std::to_string(j) + " is in no row and its cost falls");
          break;
        }
        v = ub[j];
      } else {
        v = finite_lb(lb[j]) ? lb[j] : finite_ub(ub[j]) ? ub[j] : 0.0;
      }
      fix(j, v);
      changed = true;
    }
  }
  // the reduced model
  P.row_kept = row_on;
  std::vector<int> new_row(m, -1);
  for (int i = 0; i < m; ++i)
    if (row_on[i]) {
      new_row[i] = static_cast<int>(P.row_map.size());
      P.row_map.push_back(i);
      P.rhs.push_back(rhs[i]);
      P.sense.push_back(p.sense[i]);
    }
  P.col_ptr.push_back(0);
  for (int j = 0; j < n; ++j) {
    if (!col_on[j]) continue;
    P.col_map.push_back(j);
    P.obj.push_back(p.obj ? p.obj[j] : 0.0);
    P.lb.push_back(lb[j]);
    P.ub.push_back(ub[j]);
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k)
      if (row_on[p.row_idx[k]]) {
        P.row_idx.push_back(new_row[p.row_idx[k]]);
        P.values.push_back(p.values[k]);
      }
    P.col_ptr.push_back(static_cast<int32_t>(P.row_idx.size()));
  }
  sov_model& r = P.reduced;
  std::memset(&r, 0, sizeof(r));
  r.n = static_cast<int32_t>(P.col_map.size());
  r.m = static_cast<int32_t>(P.row_map.size());
  r.maximize = p.maximize;
  r.col_ptr = P.col_ptr.data();
  r.row_idx = P.row_idx.data();
  r.values = P.values.data();
  r.obj = P.obj.data();
  r.obj_constant = constant;
  r.lb = P.lb.data();
  r.ub = P.ub.data();
  r.sense = P.sense.data();
  r.rhs = P.rhs.data();
  if (P.status < 0 && r.n == 0) {
    P.status = SOV_OPTIMAL;
    P.message = "Optimal (presolve fixed all variables).";
  }
}

}  // namespace

extern "C" {

int sov_presolve_lp(const sov_model* model, sov_presolve** out) {
  if (!model || !out || model->n < 0 || model->m < 0 || (model->n > 0 && !model->col_ptr) ||
      (model->m > 0 && (!model->sense || !model->rhs)))
    return sov::record_error(SOV_E_ARGUMENT, "presolve: bad model");
  if (model->q_col_ptr) return sov::record_error(SOV_E_UNSUPPORTED, "presolve: LPs only (the reference presolves LPs only)");
  const int nnz = model->n > 0 ? model->col_ptr[model->n] : 0;
  for (int k = 0; k < nnz; ++k)
    if (model->row_idx[k] < 0 || model->row_idx[k] >= model->m)
      return sov::record_error(SOV_E_ARGUMENT, "presolve: row index out of range");
  auto* P = new sov_presolve();
  P->orig = model;
  try {
    run(*P);
  } catch (const std::exception& e) {
    delete P;
    return sov::record_error(SOV_E_ARGUMENT, std::string("presolve: ") + e.what());
  }
  *out = P;
  return SOV_OK;
}

const sov_model* sov_presolve_reduced(const sov_presolve* P) { return P ? &P->reduced : nullptr; }

int sov_presolve_info(const sov_presolve* P, int32_t* status, int32_t* rows_removed, int32_t* cols_removed,
                      int32_t* bounds_tightened, char* message, int32_t message_len) {
  if (!P) return sov::record_error(SOV_E_ARGUMENT, "presolve: null handle");
  if (status) *status = P->status;
  if (rows_removed) *rows_removed = P->rows_removed;
  if (cols_removed) *cols_removed = P->cols_removed;
  if (bounds_tightened) *bounds_tightened = P->bounds_tightened;
  if (message && message_len > 0) std::snprintf(message, message_len, "%s", P->message.c_str());
  return SOV_OK;
}

int sov_postsolve_lp(const sov_presolve* P, const sov_result* reduced, sov_result* full) {
  if (!P || !full || (P->status < 0 && !reduced)) return sov::record_error(SOV_E_ARGUMENT, "postsolve: null argument");
  const sov_model& p = *P->orig;
  const int n = p.n, m = p.m;
  const double sign = p.maximize ? -1.0 : 1.0;
  std::vector<double> x(n), y(m, 0.0), d(n, 0.0);
  const int rn = P->reduced.n, rm = P->reduced.m;
  for (int j = 0; j < n; ++j) x[j] = std::isnan(P->fixed[j]) ? 0.0 : P->fixed[j];
  if (P->status < 0) {
    if (rn > 0 && !reduced->primal) return sov::record_error(SOV_E_ARGUMENT, "postsolve: reduced result has no primal");
    for (int k = 0; k < rn; ++k) x[P->col_map[k]] = reduced->primal[k];
    if (reduced->dual_row)
      for (int k = 0; k < rm; ++k) y[P->row_map[k]] = reduced->dual_row[k];
  }
  // reduced costs with the multipliers known so far; removed rows are filled last to first
  auto reduced_cost = [&](int j) {
    double v = sign * (p.obj ? p.obj[j] : 0.0);
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) v -= p.values[k] * y[p.row_idx[k]];
    return v;
  };
  std::vector<double> act(m, 0.0);  // row activities at x
  for (int j = 0; j < n; ++j)
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) act[p.row_idx[k]] += p.values[k] * x[j];
  for (auto it = P->removed_rows.rbegin(); it != P->removed_rows.rend(); ++it) {
    if (it->col < 0) continue;  // an empty row: multiplier 0
    const int i = it->row, j = it->col, s = p.sense[i];
    const double tol = 1e-7 * (1.0 + std::fabs(p.rhs[i]) + std::fabs(act[i]));
    if (s != SOV_EQ && std::fabs(act[i] - p.rhs[i]) > tol) continue;  // slack: multiplier 0
    double yi = reduced_cost(j) / it->a;   // y_i is still 0 here
    if (s == SOV_LE && yi > 0.0) yi = 0.0;  // minimisation form: y <= 0 on <= rows
    if (s == SOV_GE && yi < 0.0) yi = 0.0;  // y >= 0 on >= rows
    y[i] = yi;
  }
  for (int j = 0; j < n; ++j) d[j] = reduced_cost(j);
  // the result
  if (P->status < 0) {
    const sov_result keep = *full;
    *full = *reduced;
    full->primal = keep.primal;
    full->dual_col = keep.dual_col;
    full->dual_row = keep.dual_row;
    full->ipm_x = keep.ipm_x;
    full->ipm_y = keep.ipm_y;
    full->ipm_s = keep.ipm_s;
    full->diagnostics = keep.diagnostics;
    if (reduced->diagnostics && keep.diagnostics && reduced->diagnostics != keep.diagnostics)
      *keep.diagnostics = *reduced->diagnostics;
  } else {
    full->status = P->status;
    full->iterations = 0;
    full->has_objective_value = P->status == SOV_OPTIMAL ? 1 : 0;
    full->duality_gap = full->primal_residual = full->dual_residual = 0.0;
    full->n_ipm = full->m_ipm = 0;
  }
  if (full->primal) std::copy(x.begin(), x.end(), full->primal);
  if (full->dual_row) std::copy(y.begin(), y.end(), full->dual_row);
  if (full->dual_col)
    for (int j = 0; j < n; ++j) {
      // kept columns carry the engine's reduced cost; removed ones the recomputed one
      full->dual_col[j] = d[j];
    }
  if (P->status < 0 && reduced->dual_col)
    for (int k = 0; k < rn; ++k)
      if (full->dual_col) full->dual_col[P->col_map[k]] = reduced->dual_col[k];
  double obj = p.obj_constant;
  for (int j = 0; j < n; ++j) obj += (p.obj ? p.obj[j] : 0.0) * x[j];
  if (full->has_objective_value) full->objective_value = obj;
  char head[160];
  std::snprintf(head, sizeof head, "Presolve removed %d rows and %d columns, tightened %d bounds (%d passes). ",
                P->rows_removed, P->cols_removed, P->bounds_tightened, P->passes);
  const std::string tail = P->status < 0 ? std::string(reduced->message) : P->message;
  std::snprintf(full->message, sizeof(full->message), "%s%s", head, tail.c_str());
  return SOV_OK;
}

void sov_presolve_destroy(sov_presolve* P) { delete P; }

}  // extern "C"
