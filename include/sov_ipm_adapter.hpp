// sov_ipm_adapter.hpp -- header-only binding of libsovipm into the reference's C++ solver.
//
// Compiled inside the Abhishekmishra2808/sovereign tree (it includes the reference's
// "sovereign/types.hpp"); it turns a name-keyed sovereign::OptimizationModel
// (solver/core/include/sovereign/types.hpp:53-59) into the index-form sov_model of sov_ipm.h,
// calls the GPU engine, and maps the answer back into a sovereign::SolverResult
// (types.hpp:117-155) with the keys the reference's IPM publishes: primal and dual-slack values by
// variable name, row multipliers as "row_<i>", dual_certificate_space "original_model" and
// lp_diagnostics["ipm"] (solver/lp/src/interior_point.cpp:521-569).
//
// Drop-in use (solver/lp/src/lp_solver.cpp:59-62):
//     auto run_ipm = [&]() {
//       if (const char* b = std::getenv("SOVEREIGN_IPM_BACKEND"); b && std::string(b) == "b200")
//         return sovereign::b200::solve_lp(model);
//       InteriorPointOptions opt;
//       return InteriorPointSolver(opt).solve(model);
//     };
// and for QP (solver/qp/src/qp_solver.cpp:36) sovereign::b200::solve_qp(model).
#pragma once

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "sov_ipm.h"
#include "sovereign/types.hpp"

namespace sovereign {
namespace b200 {

namespace detail {

struct IndexModel {
  std::vector<int32_t> col_ptr, row_idx, q_ptr, q_idx;
  std::vector<double> values, obj, lb, ub, rhs, q_val;
  std::vector<int8_t> sense;
  sov_model view{};
};

inline IndexModel to_index(const OptimizationModel& model, bool qp) {
  IndexModel im;
  const int n = static_cast<int>(model.variables.size());
  const int m = static_cast<int>(model.constraints.size());
  std::unordered_map<std::string, int> index;
  index.reserve(static_cast<std::size_t>(n) * 2);
  for (int j = 0; j < n; ++j) index[model.variables[j].name] = j;
  im.obj.assign(n, 0.0);
  im.lb.resize(n);
  im.ub.resize(n);
  for (int j = 0; j < n; ++j) {
    im.lb[j] = model.variables[j].lower_bound;
    im.ub[j] = model.variables[j].upper_bound;
    auto it = model.objective.linear.find(model.variables[j].name);
    if (it != model.objective.linear.end()) im.obj[j] = it->second;
  }
  std::vector<std::vector<std::pair<int, double>>> cols(n);
  im.sense.resize(m);
  im.rhs.resize(m);
  for (int i = 0; i < m; ++i) {
    const Constraint& c = model.constraints[i];
    im.sense[i] = c.sense == ConstraintSense::Le ? SOV_LE : c.sense == ConstraintSense::Ge ? SOV_GE : SOV_EQ;
    im.rhs[i] = c.rhs;
    for (const auto& kv : c.linear) {
      auto it = index.find(kv.first);
      if (it == index.end()) throw std::runtime_error("Unknown variable in constraint: " + kv.first);
      cols[it->second].push_back({i, kv.second});
    }
  }
  im.col_ptr.assign(n + 1, 0);
  for (int j = 0; j < n; ++j) {
    std::sort(cols[j].begin(), cols[j].end());
    for (const auto& e : cols[j]) {
      im.row_idx.push_back(e.first);
      im.values.push_back(e.second);
    }
    im.col_ptr[j + 1] = static_cast<int32_t>(im.row_idx.size());
  }
  if (qp) {
    // stored quadratic terms q_ij (row name -> col name -> value), one CSC entry per stored term
    std::vector<std::vector<std::pair<int, double>>> qc(n);
    for (const auto& row : model.objective.quadratic) {
      auto ri = index.find(row.first);
      if (ri == index.end()) continue;
      for (const auto& col : row.second) {
        auto cj = index.find(col.first);
        if (cj == index.end()) continue;
        qc[cj->second].push_back({ri->second, col.second});
      }
    }
    im.q_ptr.assign(n + 1, 0);
    for (int j = 0; j < n; ++j) {
      for (const auto& e : qc[j]) {
        im.q_idx.push_back(e.first);
        im.q_val.push_back(e.second);
      }
      im.q_ptr[j + 1] = static_cast<int32_t>(im.q_idx.size());
    }
  }
  sov_model& v = im.view;
  v.n = n;
  v.m = m;
  v.maximize = model.sense == Sense::Maximize ? 1 : 0;
  v.col_ptr = im.col_ptr.data();
  v.row_idx = im.row_idx.data();
  v.values = im.values.data();
  v.obj = im.obj.data();
  v.obj_constant = model.objective.constant;
  v.lb = im.lb.data();
  v.ub = im.ub.data();
  v.sense = im.sense.data();
  v.rhs = im.rhs.data();
  if (qp) {
    v.q_col_ptr = im.q_ptr.data();
    v.q_row_idx = im.q_idx.data();
    v.q_values = im.q_val.data();
  }
  return im;
}

inline SolverResult to_result(const OptimizationModel& model, const sov_result& r, const std::vector<double>& x,
                              const std::vector<double>& dcol, const std::vector<double>& drow,
                              const sov_diagnostics& dg) {
  SolverResult out;
  out.status = static_cast<SolverStatus>(r.status);
  out.iterations = r.iterations;
  out.has_objective_value = r.has_objective_value != 0;
  out.objective_value = r.objective_value;
  out.duality_gap = r.duality_gap;
  out.primal_residual = r.primal_residual;
  out.dual_residual = r.dual_residual;
  out.message = r.message;
  out.runtime_seconds = r.solve_seconds;
  if (out.has_objective_value) {
    out.dual_certificate_space = "original_model";
    for (std::size_t j = 0; j < model.variables.size(); ++j) {
      out.primal[model.variables[j].name] = x[j];
      out.dual[model.variables[j].name] = dcol[j];
    }
    for (std::size_t i = 0; i < model.constraints.size(); ++i) out.dual["row_" + std::to_string(i)] = drow[i];
  }
  LpDiagnostics& d = out.lp_diagnostics["ipm"];
  d.scaling_applied = dg.scaling_applied != 0;
  d.coefficient_min_abs_before = dg.coefficient_min_abs_before;
  d.coefficient_max_abs_before = dg.coefficient_max_abs_before;
  d.coefficient_min_abs_after = dg.coefficient_min_abs_after;
  d.coefficient_max_abs_after = dg.coefficient_max_abs_after;
  d.refactorizations = dg.refactorizations;
  for (int k = 0; k < dg.history_len; ++k) {
    d.objective_history_iterations.push_back(dg.history_iterations[k]);
    d.objective_history.push_back(dg.objective_history[k]);
    d.gap_history_iterations.push_back(dg.history_iterations[k]);
    d.gap_history.push_back(dg.gap_history[k]);
    d.mu_history.push_back(dg.mu_history[k]);
  }
  for (int k = 0; k < dg.step_history_len; ++k) {
    d.primal_step_history.push_back(dg.primal_step_history[k]);
    d.dual_step_history.push_back(dg.dual_step_history[k]);
  }
  d.stall_iteration = dg.stall_iteration;
  d.stall_gap = dg.stall_gap;
  d.stall_mu = dg.stall_mu;
  d.stall_primal_step = dg.stall_primal_step;
  d.stall_dual_step = dg.stall_dual_step;
  d.final_primal_residual = r.primal_residual;
  d.final_dual_residual = r.dual_residual;
  d.final_gap = r.duality_gap;
  d.basis_state = "interior_point";
  d.stop_reason = r.message;
  return out;
}

inline SolverResult solve(const OptimizationModel& model, bool qp, const sov_options* opt) {
  try {
    IndexModel im = to_index(model, qp);
    std::vector<double> x(im.view.n), dcol(im.view.n), drow(im.view.m);
    sov_diagnostics dg;
    std::memset(&dg, 0, sizeof(dg));
    sov_result r;
    std::memset(&r, 0, sizeof(r));
    r.primal = x.data();
    r.dual_col = dcol.data();
    r.dual_row = drow.data();
    r.diagnostics = &dg;
    const int rc = qp ? sov_qp_solve(&im.view, opt, &r) : sov_lp_solve(&im.view, opt, &r);
    if (rc != SOV_OK && r.message[0] == '\0')
      std::snprintf(r.message, sizeof(r.message), "%s error: %s", qp ? "QP-IPM" : "IPM", sov_last_error());
    return to_result(model, r, x, dcol, drow, dg);
  } catch (const std::exception& ex) {
    // same convention as InteriorPointSolver::solve (interior_point.cpp:748-756)
    SolverResult r;
    r.status = SolverStatus::Error;
    r.message = std::string(qp ? "QP-IPM error: " : "IPM error: ") + ex.what();
    return r;
  }
}

}  // namespace detail

inline SolverResult solve_lp(const OptimizationModel& model, const sov_options* opt = nullptr) {
  return detail::solve(model, false, opt);
}

inline SolverResult solve_qp(const OptimizationModel& model, const sov_options* opt = nullptr) {
  return detail::solve(model, true, opt);
}

}  // namespace b200
}  // namespace sovereign
