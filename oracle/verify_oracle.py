"""TEST INFRASTRUCTURE ONLY -- CPU restatement of the solution certificate.

Primal figures restate sovereign::SolutionVerifier::verify (solver/core/src/verifier.cpp:10-150):
bound violation max(lb - x, x - ub) (:52-54), row violation by sense (:86-98), the objective
recomputed from the model (:67-82), and the verdict's issues (:17-38, :100-148). The dual figures
(reduced-cost and row-dual signs, dual objective, relative gap) restate the definitions written in
include/sov_ipm.h for sov_certificate. Exact sums (math.fsum) stand in for the GPU's double-double.
"""
from __future__ import annotations

import math

import numpy as np

LE, GE, EQ = 0, 1, 2


def certificate(model, primal, dual_row, status, objective_value, duality_gap, has_objective=True, tol=1e-6):
    n, m = model.n, model.m
    x = np.asarray(primal, dtype=np.float64)
    y = np.asarray(dual_row, dtype=np.float64)
    lb = model.lb if model.lb is not None else np.zeros(n)
    ub = model.ub if model.ub is not None else np.full(n, 1e30)
    sign = -1.0 if model.maximize else 1.0
    A = np.zeros((m, n))
    for j in range(n):
        for k in range(model.col_ptr[j], model.col_ptr[j + 1]):
            A[model.row_idx[k], j] += model.values[k]
    Qs = np.zeros((n, n))  # symmetric form of the stored terms
    if model.q_col_ptr is not None:
        for j in range(n):
            for k in range(model.q_col_ptr[j], model.q_col_ptr[j + 1]):
                i = model.q_row_idx[k]
                Qs[i, j] += 0.5 * model.q_values[k]
                Qs[j, i] += 0.5 * model.q_values[k]
    bound = max(0.0, float(np.max(np.maximum(lb - x, x - ub)))) if n else 0.0
    act = np.array([math.fsum(A[i] * x) for i in range(m)])
    viol = np.where(model.sense == LE, act - model.rhs, np.where(model.sense == GE, model.rhs - act,
                                                                 np.abs(act - model.rhs)))
    cons = max(0.0, float(np.max(viol))) if m else 0.0
    qx = Qs @ x
    obj = math.fsum(list(model.obj * x) + list(0.5 * x * qx) + [model.obj_constant])
    d = sign * model.obj + sign * qx - A.T @ y
    has_lo, has_hi = lb > -1e29, ub < 1e29
    dual_viol = 0.0
    bterm = []
    for j in range(n):
        if has_lo[j] and has_hi[j]:
            bterm.append((lb[j] if d[j] > 0 else ub[j]) * d[j])
        elif has_lo[j]:
            dual_viol = max(dual_viol, -d[j])
            bterm.append(lb[j] * max(d[j], 0.0))
        elif has_hi[j]:
            dual_viol = max(dual_viol, d[j])
            bterm.append(ub[j] * min(d[j], 0.0))
        else:
            dual_viol = max(dual_viol, abs(d[j]))
    for i in range(m):
        if model.sense[i] == LE:
            dual_viol = max(dual_viol, y[i])
        elif model.sense[i] == GE:
            dual_viol = max(dual_viol, -y[i])
    xqx = sign * float(x @ qx)
    dual_min = math.fsum(list(model.rhs * y) + bterm) - 0.5 * xqx + sign * model.obj_constant
    primal_min = sign * obj
    issues = 0
    if status in (8, 7, 6, 4, 5):
        issues |= 1
    elif status in (2, 3):
        issues |= 2
    else:
        if bound > tol:
            issues |= 8
        if cons > tol:
            issues |= 16
        if has_objective and abs(objective_value - obj) > tol * (1.0 + abs(obj)):
            issues |= 32
        if status == 0 and duality_gap > tol:
            issues |= 64
    return dict(max_bound_violation=bound, max_constraint_violation=cons, recomputed_objective=obj,
                dual_objective=sign * dual_min, max_dual_infeasibility=dual_viol,
                relative_gap=abs(primal_min - dual_min) / (1.0 + abs(primal_min)), issues=issues,
                is_valid=issues == 0)
