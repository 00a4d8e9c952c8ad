// The reference-side adapter (include/sov_ipm_adapter.hpp) on a GPU, against the reference's own
// solvers in the same process: sovereign::b200::solve_lp / solve_qp / solve_lp_batch /
// solve_lp_family / solve_branch_children on name-keyed OptimizationModels, compared with InteriorPointSolver and
// QpInteriorPointSolver (solver/lp/src/interior_point.cpp:747-757,
// solver/qp/src/qp_interior_point.cpp:3123-3186) on the same models: status, objective (1e-8
// relative), the key sets and values of the name-keyed primal and dual maps ("row_<i>" for rows),
// dual_certificate_space and lp_diagnostics["ipm"] (scaling flags and coefficient ranges exactly).
// Built by oracle/Makefile next to the reference library (it compiles the reference's sources);
// run by tests/test_adapter.py. Prints "failures N". With --reference-only (no GPU needed) it
// checks only that the reference solves every model of the comparison to OPTIMAL.
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

#include "sov_ipm_adapter.hpp"
#include "sovereign/interior_point.hpp"
#include "sovereign/qp_interior_point.hpp"
#include "sovereign/verifier.hpp"

using namespace sovereign;

namespace {

int failures = 0;

void fail(const std::string& what) {
  std::printf("FAIL %s\n", what.c_str());
  ++failures;
}

double rel(double a, double b) { return std::fabs(a - b) / std::max(1.0, std::fabs(b)); }

OptimizationModel transport(int ns, int nt, unsigned seed) {
  std::mt19937 rng(seed);
  OptimizationModel m;
  m.problem_type = ProblemType::LP;
  m.sense = Sense::Minimize;
  std::vector<double> sup(ns), dem(nt);
  double total = 0.0;
  for (auto& s : sup) total += (s = 10 + rng() % 91);
  double left = total;
  for (int j = 0; j < nt; ++j) {
    dem[j] = j + 1 < nt ? std::floor(total / nt) : left;
    left -= dem[j];
  }
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < nt; ++j) {
      Variable v;
      v.name = "ship_" + std::to_string(i) + "_" + std::to_string(j);
      m.variables.push_back(v);
      m.objective.linear[v.name] = 1.0 + (rng() % 9900) / 100.0;
    }
  for (int i = 0; i < ns; ++i) {
    Constraint c;
    c.name = "supply_" + std::to_string(i);
    c.sense = ConstraintSense::Eq;
    c.rhs = sup[i];
    for (int j = 0; j < nt; ++j) c.linear["ship_" + std::to_string(i) + "_" + std::to_string(j)] = 1.0;
    m.constraints.push_back(c);
  }
  for (int j = 0; j < nt; ++j) {
    Constraint c;
    c.name = "demand_" + std::to_string(j);
    c.sense = ConstraintSense::Eq;
    c.rhs = dem[j];
    for (int i = 0; i < ns; ++i) c.linear["ship_" + std::to_string(i) + "_" + std::to_string(j)] = 1.0;
    m.constraints.push_back(c);
  }
  return m;
}

// A random LP with mixed row senses, shifted lower bounds, some upper bounds and maximisation;
// feasible at x0 and bounded (costs from a dual point), so it has an optimum.
OptimizationModel random_lp(int rows, int cols, unsigned seed, bool maximize) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  std::normal_distribution<double> g(0.0, 1.0);
  OptimizationModel m;
  m.problem_type = ProblemType::LP;
  m.sense = maximize ? Sense::Maximize : Sense::Minimize;
  std::vector<double> x0(cols);
  for (int j = 0; j < cols; ++j) {
    Variable v;
    v.name = "v" + std::to_string(j);
    v.lower_bound = (j % 5 == 0) ? -1.0 : 0.0;
    v.upper_bound = (j % 7 == 0) ? 3.0 : 1e30;
    x0[j] = v.lower_bound + 0.2 + 0.6 * u(rng);
    m.variables.push_back(v);
  }
  std::vector<std::vector<std::pair<int, double>>> a(rows);
  for (int j = 0; j < cols; ++j)
    for (int k = 0; k < 3; ++k) a[rng() % rows].push_back({j, g(rng)});
  std::vector<double> y(rows), cost(cols, 0.0);
  for (int i = 0; i < rows; ++i) {
    Constraint c;
    c.name = "c" + std::to_string(i);
    double ax = 0.0;
    for (auto [j, v] : a[i]) {
      c.linear["v" + std::to_string(j)] += v;
      ax += v * x0[j];
    }
    const int kind = i % 3;
    c.sense = kind == 0 ? ConstraintSense::Eq : kind == 1 ? ConstraintSense::Le : ConstraintSense::Ge;
    c.rhs = kind == 0 ? ax : kind == 1 ? ax + 0.5 : ax - 0.5;
    y[i] = kind == 0 ? g(rng) : kind == 1 ? -u(rng) : u(rng);
    for (auto [j, v] : a[i]) cost[j] += v * y[i];
    m.constraints.push_back(c);
  }
  for (int j = 0; j < cols; ++j) {
    const double cj = cost[j] + 0.1 + u(rng);
    m.objective.linear["v" + std::to_string(j)] = maximize ? -cj : cj;
  }
  return m;
}

OptimizationModel portfolio(int assets, unsigned seed) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  OptimizationModel m;
  m.problem_type = ProblemType::QP;
  m.sense = Sense::Minimize;
  Constraint budget;
  budget.name = "budget";
  budget.sense = ConstraintSense::Eq;
  budget.rhs = 1.0;
  Constraint ret;
  ret.name = "return";
  ret.sense = ConstraintSense::Ge;
  ret.rhs = 0.05;
  for (int j = 0; j < assets; ++j) {
    Variable v;
    v.name = "w" + std::to_string(j);
    v.upper_bound = 0.4;
    m.variables.push_back(v);
    m.objective.quadratic[v.name][v.name] = 0.02 + 0.2 * u(rng);
    budget.linear[v.name] = 1.0;
    ret.linear[v.name] = 0.01 + 0.1 * u(rng);
  }
  m.constraints.push_back(budget);
  m.constraints.push_back(ret);
  return m;
}

void compare(const std::string& name, const OptimizationModel& m, const SolverResult& got, const SolverResult& want,
             double value_tol) {
  if (got.status != want.status)
    return fail(name + ": status " + std::to_string(int(got.status)) + " vs " + std::to_string(int(want.status)));
  if (want.status != SolverStatus::Optimal) return fail(name + ": reference not optimal");
  if (rel(got.objective_value, want.objective_value) > 1e-8)
    return fail(name + ": objective " + std::to_string(got.objective_value) + " vs " +
                std::to_string(want.objective_value));
  if (got.primal.size() != want.primal.size()) return fail(name + ": primal map sizes");
  for (const auto& kv : want.primal) {
    auto it = got.primal.find(kv.first);
    if (it == got.primal.end()) return fail(name + ": missing primal " + kv.first);
    if (std::fabs(it->second - kv.second) > value_tol * (1.0 + std::fabs(kv.second)))
      return fail(name + ": primal " + kv.first + " " + std::to_string(it->second) + " vs " + std::to_string(kv.second));
  }
  // row multipliers are not unique where the primal optimum is degenerate (a transportation LP's
  // rows are dependent): the keys must match and the GPU certificate must close the gap with them
  for (const auto& kv : want.dual)
    if (kv.first.rfind("row_", 0) == 0 && !got.dual.count(kv.first)) return fail(name + ": missing dual " + kv.first);
  for (std::size_t i = 0; i < m.constraints.size(); ++i)
    if (!got.dual.count("row_" + std::to_string(i))) return fail(name + ": no row_" + std::to_string(i));
  if (got.dual_certificate_space != want.dual_certificate_space) return fail(name + ": dual_certificate_space");
  const auto g = got.lp_diagnostics.find("ipm"), w = want.lp_diagnostics.find("ipm");
  if ((g == got.lp_diagnostics.end()) != (w == want.lp_diagnostics.end())) return fail(name + ": lp_diagnostics");
  if (w != want.lp_diagnostics.end()) {
    const LpDiagnostics &a = g->second, &b = w->second;
    if (a.scaling_applied != b.scaling_applied || a.coefficient_min_abs_before != b.coefficient_min_abs_before ||
        a.coefficient_max_abs_before != b.coefficient_max_abs_before ||
        a.coefficient_min_abs_after != b.coefficient_min_abs_after ||
        a.coefficient_max_abs_after != b.coefficient_max_abs_after)
      return fail(name + ": scaling diagnostics");
    if (a.final_gap > 1e-8) return fail(name + ": final gap");
  }
  // the GPU certificate against the reference's SolutionVerifier on the same answer
  sov_certificate cert;
  const VerificationResult vg = b200::verify(m, got, 1e-6, &cert), vr = SolutionVerifier().verify(m, got);
  if (cert.relative_gap > 1e-7)
    return fail(name + ": the published multipliers leave a relative gap of " + std::to_string(cert.relative_gap));
  auto near = [](double a, double b) { return std::fabs(a - b) <= 1e-12 * std::max(1.0, std::fabs(b)); };
  if (vg.is_valid != vr.is_valid || vg.issues.size() != vr.issues.size() ||
      !near(vg.max_bound_violation, vr.max_bound_violation) ||
      !near(vg.max_constraint_violation, vr.max_constraint_violation) ||
      !near(vg.recomputed_objective, vr.recomputed_objective))
    return fail(name + ": GPU verification differs from SolutionVerifier (" + vg.message + " / " + vr.message + ")");
  std::printf("ok %s: %s objective %.12g (reference %.12g), %d vs %d iterations\n", name.c_str(),
              got.message.substr(0, 40).c_str(), got.objective_value, want.objective_value,
              static_cast<int>(got.iterations), static_cast<int>(want.iterations));
}

}  // namespace

int main(int argc, char** argv) {
  const InteriorPointSolver ref_lp{InteriorPointOptions{}};
  const bool reference_only = argc > 1 && std::string(argv[1]) == "--reference-only";
  if (reference_only) {  // the models of the comparison, reference side only
    for (const auto& m : {transport(12, 15, 1), random_lp(60, 150, 2, false), random_lp(90, 200, 3, true),
                          random_lp(50, 120, 31, false)})
      if (ref_lp.solve(m).status != SolverStatus::Optimal) fail("reference LP not optimal");
    for (int k = 0; k < 6; ++k) {
      const OptimizationModel m = k % 2 ? random_lp(40 + k, 90, 10 + k, false) : transport(5 + k, 6, 20 + k);
      if (ref_lp.solve(m).status != SolverStatus::Optimal) fail("reference node LP not optimal");
    }
    for (int k = 0; k < 8; ++k)
      if (ref_lp.solve(transport(12, 15, 40 + k)).status != SolverStatus::Optimal) fail("reference family LP not optimal");
    if (QpInteriorPointSolver(QpInteriorPointOptions{}).solve(portfolio(30, 4)).status != SolverStatus::Optimal)
      fail("reference QP not optimal");
    std::printf("failures %d\n", failures);
    return failures == 0 ? 0 : 1;
  }
  // single LPs and QPs
  std::vector<std::pair<std::string, OptimizationModel>> lps = {
      {"transport 12x15", transport(12, 15, 1)},
      {"random 60x150", random_lp(60, 150, 2, false)},
      {"random 90x200 max", random_lp(90, 200, 3, true)},
  };
  for (const auto& [name, m] : lps) compare(name, m, b200::solve_lp(m), ref_lp.solve(m), 1e-5);
  {
    const OptimizationModel q = portfolio(30, 4);
    compare("portfolio 30", q, b200::solve_qp(q), QpInteriorPointSolver(QpInteriorPointOptions{}).solve(q), 1e-4);
  }
  // a perturbed answer: both verifiers reject it with the same issues
  {
    const OptimizationModel m = transport(8, 9, 5);
    SolverResult r = b200::solve_lp(m);
    r.primal[m.variables[0].name] = -0.01;
    r.objective_value += 1.0;
    const VerificationResult vg = b200::verify(m, r), vr = SolutionVerifier().verify(m, r);
    if (vg.is_valid || vr.is_valid || vg.issues.size() != vr.issues.size())
      fail("perturbed answer: " + std::to_string(vg.issues.size()) + " vs " + std::to_string(vr.issues.size()) +
           " issues");
    for (std::size_t k = 0; k < vg.issues.size() && k < vr.issues.size(); ++k)
      if (vg.issues[k].substr(0, 20) != vr.issues[k].substr(0, 20)) fail("issue text: " + vg.issues[k] + " / " + vr.issues[k]);
  }
  // node LPs in one batch (one of them refers to an unknown variable: an error for it alone)
  {
    std::vector<OptimizationModel> nodes;
    for (int k = 0; k < 6; ++k) nodes.push_back(k % 2 ? random_lp(40 + k, 90, 10 + k, false) : transport(5 + k, 6, 20 + k));
    OptimizationModel bad = transport(3, 3, 7);
    bad.constraints[0].linear["nope"] = 1.0;
    nodes.push_back(bad);
    const auto got = b200::solve_lp_batch(nodes);
    for (std::size_t k = 0; k + 1 < nodes.size(); ++k)
      compare("batch node " + std::to_string(k), nodes[k], got[k], ref_lp.solve(nodes[k]), 1e-5);
    const SolverResult want_bad = ref_lp.solve(bad);
    if (got.back().status != SolverStatus::Error || got.back().message != want_bad.message)
      fail("batch error model: " + got.back().message + " vs " + want_bad.message);
  }
  // one parametric family: transport LPs of one shape with their own costs and supplies, in one
  // family call; then a set whose shapes differ, which the family call refuses for every LP
  {
    std::vector<OptimizationModel> fam;
    for (int k = 0; k < 8; ++k) fam.push_back(transport(12, 15, 40 + k));
    const auto got = b200::solve_lp_family(fam);
    for (std::size_t k = 0; k < fam.size(); ++k)
      compare("family member " + std::to_string(k), fam[k], got[k], ref_lp.solve(fam[k]), 1e-5);
    const auto mixed = b200::solve_lp_family({transport(5, 6, 1), transport(6, 6, 2)});
    for (const auto& r : mixed)
      if (r.status != SolverStatus::Error || r.message.find("does not share") == std::string::npos)
        fail("mixed family: " + r.message);
  }
  // strong-branching children of a relaxation at a fractional point
  {
    const OptimizationModel relax = random_lp(50, 120, 31, false);
    const SolverResult root = ref_lp.solve(relax);
    std::vector<int> cands;
    for (int j = 0; j < static_cast<int>(relax.variables.size()) && cands.size() < 8; ++j) {
      const double v = root.primal.at(relax.variables[j].name);
      if (v - std::floor(v) > 0.05 && std::ceil(v) - v > 0.05) cands.push_back(j);
    }
    if (cands.size() < 2) fail("too few fractional candidates");
    const auto kids = b200::solve_branch_children(relax, cands, root.primal);
    for (std::size_t c = 0; c < cands.size(); ++c) {
      const int i = cands[c];
      const double v = root.primal.at(relax.variables[i].name);
      OptimizationModel down = relax, up = relax;
      down.variables[i].upper_bound = std::min(down.variables[i].upper_bound, std::floor(v));
      up.variables[i].lower_bound = std::max(up.variables[i].lower_bound, std::ceil(v));
      const SolverResult rd = ref_lp.solve(down), ru = ref_lp.solve(up);
      if (kids[c].var != i) fail("child order");
      // children may be infeasible; then only the status has to agree
      if (rd.status == SolverStatus::Optimal) compare("down " + std::to_string(i), down, kids[c].down, rd, 1e-4);
      else if (kids[c].down.status == SolverStatus::Optimal) fail("down child optimal where the reference is not");
      if (ru.status == SolverStatus::Optimal) compare("up " + std::to_string(i), up, kids[c].up, ru, 1e-4);
      else if (kids[c].up.status == SolverStatus::Optimal) fail("up child optimal where the reference is not");
    }
  }
  std::printf("failures %d\n", failures);
  return failures == 0 ? 0 : 1;
}
