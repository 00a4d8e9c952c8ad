// sov_ipm_adapter.hpp -- header-only binding of libsovipm into the reference's C++ solver.
//
// Compiled inside the Abhishekmishra2808/sovereign tree (it includes the reference's
// "sovereign/types.hpp"); it turns a name-keyed sovereign::OptimizationModel
// (solver/core/include/sovereign/types.hpp:53-59) into the index-form sov_model of sov_ipm.h,
// calls the GPU engine, and maps the answer back into a sovereign::SolverResult
// (types.hpp:117-155) with the keys the reference's IPM publishes: primal and dual-slack values by
// variable name, row multipliers as "row_<i>", dual_certificate_space "original_model" and
// lp_diagnostics["ipm"] (solver/lp/src/interior_point.cpp:521-569); for a QP, the keys of the
// reference's QP-IPM (row multipliers of the upper-bound rows included, no certificate space).
//
// Drop-in use (solver/lp/src/lp_solver.cpp:59-62):
//     auto run_ipm = [&]() {
//       if (const char* b = std::getenv("SOVEREIGN_IPM_BACKEND"); b && std::string(b) == "b200")
//         return sovereign::b200::solve_lp(model);
//       InteriorPointOptions opt;
//       return InteriorPointSolver(opt).solve(model);
//     };
// and for QP (solver/qp/src/qp_solver.cpp:36) sovereign::b200::solve_qp(model).
//
// Batched callers (no reference counterpart for the batching itself):
//   solve_lp_batch(models)        N independent LPs in one sov_lp_solve_batch call, in place of N
//                                 InteriorPointSolver::solve calls (the node LPs of a
//                                 branch-and-bound round, solver/milp/src/branch_and_bound.cpp:497)
//   verify(model, result, tol)    SolutionVerifier::verify (solver/core/src/verifier.cpp:10-150)
//                                 computed on the GPU by sov_verify_solution, for an answer
//                                 accepted without a simplex crossover; also returns the dual side
//   solve_branch_children(relax, candidates, x)
//                                 the down/up children of strong branching
//                                 (branch_and_bound.cpp:726-779, 829-856: ub = min(ub, floor v),
//                                 lb = max(lb, ceil v)) for every candidate, all in one call
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
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

// qp: the QP solver's result maps (qp_interior_point.cpp): the general QP-IPM publishes the dual
// slack of every variable under its name and the multiplier of every IPM row -- the model's rows,
// then one per finite upper bound -- as "row_<i>" (capture_diagnostics, :2862-2870), and sets no
// certificate space; the structured path for the convex-sequence shape publishes the model's rows
// only (:2198-2202); neither records lp_diagnostics. ipm_y: the final IPM multipliers (m_ipm), or
// empty.
inline SolverResult to_result(const OptimizationModel& model, const sov_result& r, const std::vector<double>& x,
                              const std::vector<double>& dcol, const std::vector<double>& drow,
                              const sov_diagnostics& dg, bool qp = false,
                              const std::vector<double>& ipm_y = std::vector<double>()) {
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
    if (!qp) out.dual_certificate_space = "original_model";
    const bool structured = qp && dg.structured_qp;
    for (std::size_t j = 0; j < model.variables.size(); ++j) {
      out.primal[model.variables[j].name] = x[j];
      if (!structured) out.dual[model.variables[j].name] = dcol[j];
    }
    for (std::size_t i = 0; i < model.constraints.size(); ++i) out.dual["row_" + std::to_string(i)] = drow[i];
    if (qp && !structured)
      for (std::size_t i = model.constraints.size(); i < ipm_y.size(); ++i)
        out.dual["row_" + std::to_string(i)] = ipm_y[i];
  }
  if (qp) return out;  // the QP solver records no lp_diagnostics
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
    std::vector<double> x(im.view.n), dcol(im.view.n), drow(im.view.m), ipm_y;
    sov_diagnostics dg;
    std::memset(&dg, 0, sizeof(dg));
    sov_result r;
    std::memset(&r, 0, sizeof(r));
    r.primal = x.data();
    r.dual_col = dcol.data();
    r.dual_row = drow.data();
    r.diagnostics = &dg;
    int32_t n_ipm = 0, m_ipm = 0;
    if (qp && sov_ipm_dims(&im.view, 1, &n_ipm, &m_ipm) == SOV_OK && m_ipm > 0) {
      ipm_y.assign(m_ipm, 0.0);
      r.ipm_y = ipm_y.data();
    }
    const int rc = qp ? sov_qp_solve(&im.view, opt, &r) : sov_lp_solve(&im.view, opt, &r);
    if (rc != SOV_OK && r.message[0] == '\0')
      std::snprintf(r.message, sizeof(r.message), "%s error: %s", qp ? "QP-IPM" : "IPM", sov_last_error());
    if (r.m_ipm != m_ipm) ipm_y.clear();
    return to_result(model, r, x, dcol, drow, dg, qp, ipm_y);
  } catch (const std::exception& ex) {
    // same convention as InteriorPointSolver::solve (interior_point.cpp:748-756)
    SolverResult r;
    r.status = SolverStatus::Error;
    r.message = std::string(qp ? "QP-IPM error: " : "IPM error: ") + ex.what();
    return r;
  }
}

// Output arrays of one LP of a batch.
struct BatchSlot {
  std::vector<double> x, dcol, drow;
  sov_diagnostics dg;
  sov_result r;
  void bind(int n, int m) {
    x.assign(n, 0.0);
    dcol.assign(n, 0.0);
    drow.assign(m, 0.0);
    std::memset(&dg, 0, sizeof(dg));
    std::memset(&r, 0, sizeof(r));
    r.primal = x.data();
    r.dual_col = dcol.data();
    r.dual_row = drow.data();
    r.diagnostics = &dg;
  }
};

inline SolverResult error_result(const std::string& what) {
  SolverResult r;
  r.status = SolverStatus::Error;
  r.message = "IPM error: " + what;
  return r;
}

// One sov_lp_solve_batch (or, with `family`, sov_lp_solve_family) call over `views` (model k of
// the caller is views[k]'s source); a failed call marks every LP of it with the recorded error.
inline std::vector<SolverResult> run_batch(const std::vector<const OptimizationModel*>& sources,
                                           std::vector<sov_model>& views, const sov_options* opt,
                                           bool family = false) {
  const int count = static_cast<int>(views.size());
  std::vector<BatchSlot> slots(count);
  std::vector<sov_result> res(count);
  for (int k = 0; k < count; ++k) {
    slots[k].bind(views[k].n, views[k].m);
    res[k] = slots[k].r;
  }
  std::vector<SolverResult> out;
  out.reserve(count);
  int rc = SOV_OK;
  if (count > 0)
    rc = family ? sov_lp_solve_family(count, views.data(), opt, 0, res.data())
                : sov_lp_solve_batch(count, views.data(), opt, 0, res.data());
  for (int k = 0; k < count; ++k) {
    if (rc != SOV_OK) {
      out.push_back(error_result(sov_last_error()));
      continue;
    }
    out.push_back(to_result(*sources[k], res[k], slots[k].x, slots[k].dcol, slots[k].drow, slots[k].dg));
  }
  return out;
}

// Converts every model, solves those that converted in one batch or family call and puts each
// result at its model's index.
inline std::vector<SolverResult> solve_many(const std::vector<OptimizationModel>& models, const sov_options* opt,
                                            bool family) {
  std::vector<SolverResult> out(models.size());
  std::vector<detail::IndexModel> ims;
  std::vector<std::size_t> at;
  ims.reserve(models.size());
  for (std::size_t k = 0; k < models.size(); ++k) {
    try {
      ims.push_back(detail::to_index(models[k], false));
      at.push_back(k);
    } catch (const std::exception& ex) {
      out[k] = detail::error_result(ex.what());
    }
  }
  std::vector<sov_model> views;
  std::vector<const OptimizationModel*> sources;
  for (std::size_t q = 0; q < ims.size(); ++q) {
    views.push_back(ims[q].view);
    sources.push_back(&models[at[q]]);
  }
  std::vector<SolverResult> solved = detail::run_batch(sources, views, opt, family);
  for (std::size_t q = 0; q < at.size(); ++q) out[at[q]] = std::move(solved[q]);
  return out;
}

}  // namespace detail

// N independent LPs in one batched GPU call. Results in input order; a model that cannot be
// converted (unknown variable, ...) gets SolverStatus::Error with the reference's "IPM error: ..."
// message and does not stop the others.
inline std::vector<SolverResult> solve_lp_batch(const std::vector<OptimizationModel>& models,
                                                const sov_options* opt = nullptr) {
  return detail::solve_many(models, opt, false);
}

// The LPs of one parametric family -- the same variables, constraint matrix, variable bounds and
// row senses; their own objectives and right-hand sides -- in one family call
// (sov_lp_solve_family): the shared normal matrix is analysed once and 64 LPs advance together
// per launch. Each result agrees with solve_lp's for that model within the stopping tolerance.
// A model that cannot be converted gets SolverStatus::Error as in solve_lp_batch; when the
// converted models do not share their structure, every result carries the library's error.
inline std::vector<SolverResult> solve_lp_family(const std::vector<OptimizationModel>& models,
                                                 const sov_options* opt = nullptr) {
  return detail::solve_many(models, opt, true);
}

// The two children of branching on variable `var` at LP value `value`.
struct BranchChildren {
  int var = -1;
  SolverResult down, up;
};

// Strong-branching children of one LP relaxation, all candidates in one batched call: for each
// candidate index i (into relax.variables) with LP value x.at(name), the down child
// (upper_bound = min(ub, floor v)) and the up child (lower_bound = max(lb, ceil v)), exactly the
// models pick_strong_branch / pick_reliability_branch build (branch_and_bound.cpp:758-764,
// 834-839). The constraint matrix is converted once and shared by every child.
inline std::vector<BranchChildren> solve_branch_children(const OptimizationModel& relax,
                                                         const std::vector<int>& candidates,
                                                         const std::unordered_map<std::string, double>& x,
                                                         const sov_options* opt = nullptr) {
  std::vector<BranchChildren> out(candidates.size());
  detail::IndexModel im;
  try {
    im = detail::to_index(relax, false);
  } catch (const std::exception& ex) {
    for (std::size_t c = 0; c < candidates.size(); ++c) {
      out[c].var = candidates[c];
      out[c].down = out[c].up = detail::error_result(ex.what());
    }
    return out;
  }
  const std::size_t n = relax.variables.size();
  // per child its own bounds (down, up per candidate), everything else shared
  std::vector<std::vector<double>> lb(2 * candidates.size(), im.lb), ub(2 * candidates.size(), im.ub);
  std::vector<sov_model> views;
  std::vector<const OptimizationModel*> sources;
  for (std::size_t c = 0; c < candidates.size(); ++c) {
    const int i = candidates[c];
    out[c].var = i;
    if (i < 0 || static_cast<std::size_t>(i) >= n) throw std::out_of_range("branch candidate out of range");
    const double v = x.at(relax.variables[i].name);
    ub[2 * c][i] = std::min(ub[2 * c][i], std::floor(v));
    lb[2 * c + 1][i] = std::max(lb[2 * c + 1][i], std::ceil(v));
    for (int side = 0; side < 2; ++side) {
      sov_model view = im.view;
      view.lb = lb[2 * c + side].data();
      view.ub = ub[2 * c + side].data();
      views.push_back(view);
      sources.push_back(&relax);  // same names: results map back through the relaxation
    }
  }
  std::vector<SolverResult> solved = detail::run_batch(sources, views, opt);
  for (std::size_t c = 0; c < candidates.size(); ++c) {
    out[c].down = std::move(solved[2 * c]);
    out[c].up = std::move(solved[2 * c + 1]);
  }
  return out;
}

// The verifier's checks of `result` against `model` on the GPU, as a VerificationResult with the
// verifier's messages; `cert` (optional) receives every figure, the dual side included. Integrality
// is not checked (the interior-point path solves continuous models).
inline VerificationResult verify(const OptimizationModel& model, const SolverResult& result, double tol = 1e-6,
                                 sov_certificate* cert = nullptr) {
  VerificationResult out;
  out.message = "Verifier executed.";
  sov_certificate c;
  std::memset(&c, 0, sizeof(c));
  try {
    detail::IndexModel im = detail::to_index(model, !model.objective.quadratic.empty());
    std::vector<double> x(im.view.n, 0.0), y(im.view.m, 0.0);
    for (std::size_t j = 0; j < model.variables.size(); ++j) {
      auto it = result.primal.find(model.variables[j].name);
      if (it == result.primal.end()) {
        out.issues.push_back("Missing primal value for variable " + model.variables[j].name);
      } else {
        x[j] = it->second;
      }
    }
    for (std::size_t i = 0; i < model.constraints.size(); ++i) {
      auto it = result.dual.find("row_" + std::to_string(i));
      if (it != result.dual.end()) y[i] = it->second;
    }
    sov_result r;
    std::memset(&r, 0, sizeof(r));
    r.status = static_cast<int32_t>(result.status);
    r.has_objective_value = result.has_objective_value ? 1 : 0;
    r.objective_value = result.objective_value;
    r.duality_gap = result.duality_gap;
    r.primal = x.data();
    r.dual_row = y.data();
    if (sov_verify_solution(&im.view, &r, tol, &c) != SOV_OK) {
      out.issues.push_back(std::string("GPU verification failed: ") + sov_last_error());
      out.message = "Solution failed verification.";
      return out;
    }
  } catch (const std::exception& ex) {
    out.issues.push_back(std::string("IPM error: ") + ex.what());
    out.message = "Solution failed verification.";
    return out;
  }
  if (cert) *cert = c;
  out.max_bound_violation = c.max_bound_violation;
  out.max_constraint_violation = c.max_constraint_violation;
  out.recomputed_objective = c.recomputed_objective;
  if (c.issues & SOV_CERT_NO_FEASIBLE_STATUS) {
    out.issues.push_back("Solver status does not provide a feasible primal solution: " + to_string(result.status));
    out.message = "Verification skipped for non-feasible status.";
    return out;
  }
  if (c.issues & SOV_CERT_UNCHECKABLE_STATUS) {
    out.issues.push_back("Status " + to_string(result.status) + " has no independently checkable certificate.");
    out.message = "Status claim is unverified.";
    return out;
  }
  if (c.issues & SOV_CERT_NONFINITE) out.issues.push_back("Non-finite primal value or constraint activity.");
  if (c.issues & SOV_CERT_BOUND) out.issues.push_back("Bound violation exceeds tolerance.");
  if (c.issues & SOV_CERT_CONSTRAINT) out.issues.push_back("Constraint violation exceeds tolerance.");
  if (c.issues & SOV_CERT_OBJECTIVE) {
    char buf[96];
    std::snprintf(buf, sizeof buf, "Reported objective differs from recomputed value by %g",
                  std::fabs(result.objective_value - c.recomputed_objective));
    out.issues.push_back(buf);
  }
  if (c.issues & SOV_CERT_GAP) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "OPTIMAL status contradicted by reported relative duality gap %g (tolerance %g).",
                  result.duality_gap, tol);
    out.issues.push_back(buf);
  }
  out.is_valid = out.issues.empty();
  out.message = out.is_valid ? "Solution verified." : "Solution failed verification.";
  return out;
}

inline SolverResult solve_lp(const OptimizationModel& model, const sov_options* opt = nullptr) {
  return detail::solve(model, false, opt);
}

inline SolverResult solve_qp(const OptimizationModel& model, const sov_options* opt = nullptr) {
  return detail::solve(model, true, opt);
}

}  // namespace b200
}  // namespace sovereign
