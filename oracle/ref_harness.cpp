// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// Drives the reference's own CPU interior-point solvers, compiled unmodified from the
// Abhishekmishra2808/sovereign sources by oracle/Makefile into oracle/_ref/libsovref.so:
//   sovereign::InteriorPointSolver::solve   (solver/lp/src/interior_point.cpp:747-757)
//   sovereign::QpInteriorPointSolver::solve (solver/qp/src/qp_interior_point.cpp:3123-3186)
// A sov_model (include/sov_ipm.h) is turned into a sovereign::OptimizationModel with variable j
// named "x<j>" and row i named "r<i>", exactly how a JSON model would arrive, and the
// name-keyed SolverResult is mapped back to index form. Only tests/, the smoke check and the
// CPU-baseline leg of bench.py load this library; the product never does.
#include "sov_ipm.h"

#include "sovereign/interior_point.hpp"
#include "sovereign/qp_interior_point.hpp"
#include "sovereign/types.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

using namespace sovereign;

namespace {

OptimizationModel to_model(const sov_model* p, bool qp) {
  OptimizationModel model;
  model.problem_type = qp ? ProblemType::QP : ProblemType::LP;
  model.sense = p->maximize ? Sense::Maximize : Sense::Minimize;
  model.variables.resize(static_cast<std::size_t>(p->n));
  std::vector<std::string> names(static_cast<std::size_t>(p->n));
  for (int j = 0; j < p->n; ++j) {
    names[j] = "x" + std::to_string(j);
    Variable& v = model.variables[j];
    v.name = names[j];
    v.type = VariableType::Continuous;
    v.lower_bound = p->lb ? p->lb[j] : 0.0;
    v.upper_bound = p->ub ? p->ub[j] : 1e30;
    if (p->obj && p->obj[j] != 0.0) model.objective.linear[names[j]] = p->obj[j];
  }
  model.objective.constant = p->obj_constant;
  model.constraints.resize(static_cast<std::size_t>(p->m));
  for (int i = 0; i < p->m; ++i) {
    Constraint& c = model.constraints[i];
    c.name = "r" + std::to_string(i);
    c.sense = p->sense[i] == SOV_LE ? ConstraintSense::Le
              : p->sense[i] == SOV_GE ? ConstraintSense::Ge
                                      : ConstraintSense::Eq;
    c.rhs = p->rhs[i];
  }
  for (int j = 0; j < p->n; ++j) {
    for (int k = p->col_ptr[j]; k < p->col_ptr[j + 1]; ++k) {
      model.constraints[p->row_idx[k]].linear[names[j]] += p->values[k];
    }
  }
  if (qp && p->q_col_ptr) {
    for (int j = 0; j < p->n; ++j) {
      for (int k = p->q_col_ptr[j]; k < p->q_col_ptr[j + 1]; ++k) {
        model.objective.quadratic[names[p->q_row_idx[k]]][names[j]] += p->q_values[k];
      }
    }
  }
  return model;
}

void from_result(const SolverResult& r, const sov_model* p, sov_result* out) {
  out->status = static_cast<int32_t>(r.status);
  out->iterations = static_cast<int32_t>(r.iterations);
  out->has_objective_value = r.has_objective_value ? 1 : 0;
  out->objective_value = r.objective_value;
  out->duality_gap = r.duality_gap;
  out->primal_residual = r.primal_residual;
  out->dual_residual = r.dual_residual;
  if (out->primal) {
    for (int j = 0; j < p->n; ++j) {
      auto it = r.primal.find("x" + std::to_string(j));
      out->primal[j] = it == r.primal.end() ? 0.0 : it->second;
    }
  }
  if (out->dual_col) {
    for (int j = 0; j < p->n; ++j) {
      auto it = r.dual.find("x" + std::to_string(j));
      out->dual_col[j] = it == r.dual.end() ? 0.0 : it->second;
    }
  }
  if (out->dual_row) {
    for (int i = 0; i < p->m; ++i) {
      auto it = r.dual.find("row_" + std::to_string(i));
      out->dual_row[i] = it == r.dual.end() ? 0.0 : it->second;
    }
  }
  auto d = r.lp_diagnostics.find("ipm");
  if (out->diagnostics && d != r.lp_diagnostics.end()) {
    const LpDiagnostics& g = d->second;
    sov_diagnostics* o = out->diagnostics;
    o->scaling_applied = g.scaling_applied ? 1 : 0;
    o->coefficient_min_abs_before = g.coefficient_min_abs_before;
    o->coefficient_max_abs_before = g.coefficient_max_abs_before;
    o->coefficient_min_abs_after = g.coefficient_min_abs_after;
    o->coefficient_max_abs_after = g.coefficient_max_abs_after;
    o->refactorizations = static_cast<int32_t>(g.refactorizations);
    o->history_len = static_cast<int32_t>(std::min<std::size_t>(g.gap_history.size(), SOV_HISTORY_MAX));
    for (int k = 0; k < o->history_len; ++k) {
      o->history_iterations[k] = g.gap_history_iterations[k];
      o->gap_history[k] = g.gap_history[k];
      o->mu_history[k] = g.mu_history[k];
      o->objective_history[k] = g.objective_history[k];
    }
    o->step_history_len = static_cast<int32_t>(std::min<std::size_t>(g.primal_step_history.size(), SOV_HISTORY_MAX));
    for (int k = 0; k < o->step_history_len; ++k) {
      o->primal_step_history[k] = g.primal_step_history[k];
      o->dual_step_history[k] = g.dual_step_history[k];
    }
    o->stall_iteration = g.stall_iteration;
    o->stall_gap = g.stall_gap;
    o->stall_mu = g.stall_mu;
  }
  std::snprintf(out->message, sizeof(out->message), "%s", r.message.c_str());
}

}  // namespace

extern "C" {

// One solve through the reference; qp = 0 -> InteriorPointSolver, 1 -> QpInteriorPointSolver.
// max_iterations <= 0 keeps the reference default. Returns the solve time in seconds.
double ref_solve(const sov_model* p, int32_t qp, int32_t max_iterations, sov_result* out) {
  const OptimizationModel model = to_model(p, qp != 0);
  auto t0 = std::chrono::steady_clock::now();
  SolverResult r;
  if (qp) {
    QpInteriorPointOptions o;
    if (max_iterations > 0) o.max_iterations = max_iterations;
    r = QpInteriorPointSolver(o).solve(model);
  } else {
    InteriorPointOptions o;
    if (max_iterations > 0) o.max_iterations = max_iterations;
    r = InteriorPointSolver(o).solve(model);
  }
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  from_result(r, p, out);
  out->solve_seconds = secs;
  return secs;
}

// count LPs solved with InteriorPointSolver on `threads` host threads (0 = all cores). Models
// are built before the clock starts; the returned wall time covers only the solve calls, the
// way a caller holding OptimizationModels would see them. objective/iterations/status are
// written per LP when the arrays are non-null.
double ref_solve_many(int32_t count, const sov_model* ps, int32_t threads, double* objective,
                      int32_t* iterations, int32_t* status) {
  std::vector<OptimizationModel> models;
  models.reserve(static_cast<std::size_t>(count));
  for (int i = 0; i < count; ++i) models.push_back(to_model(&ps[i], false));
  int t = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
  t = std::max(1, std::min(t, count));
  std::atomic<int> next{0};
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (int w = 0; w < t; ++w) {
    pool.emplace_back([&]() {
      for (int i = next.fetch_add(1); i < count; i = next.fetch_add(1)) {
        const SolverResult r = InteriorPointSolver(InteriorPointOptions{}).solve(models[i]);
        if (objective) objective[i] = r.objective_value;
        if (iterations) iterations[i] = static_cast<int32_t>(r.iterations);
        if (status) status[i] = static_cast<int32_t>(r.status);
      }
    });
  }
  for (auto& th : pool) th.join();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int32_t ref_hardware_threads() { return static_cast<int32_t>(std::thread::hardware_concurrency()); }

}  // extern "C"
