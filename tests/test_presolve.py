"""LP presolve and postsolve in index form (sov_presolve_lp / sov_postsolve_lp /
sov_lp_solve_presolved).

* CPU: the reduced model solved by the oracle restatement and mapped back reproduces the
  reference's answer on the original model (objective to 1e-9), and the recovered row multipliers
  and reduced costs form a dual certificate (the restated SolutionVerifier plus dual checks) that
  closes the gap; decided cases (infeasible, unbounded, everything fixed) need no solve.
* GPU: the one-call presolved solve meets the reference's objective and passes the GPU
  certificate."""
import dataclasses

import numpy as np
import pytest

import oracle
from oracle import verify_oracle
from sovereign_b200 import abi, problems as P
from sovereign_b200.ipm import Presolved, solve_presolved, verify_solution


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_presolve_postsolve_with_oracle(seed):
    mdl = P.presolve_lp_example(60, 200, seed)
    want = oracle.solve(mdl, kind="reference")
    pre = Presolved(mdl)
    assert pre.status is None and pre.rows_removed >= 10 and pre.cols_removed >= 4
    assert pre.reduced.n < mdl.n and pre.reduced.m < mdl.m
    back = pre.postsolve(oracle.solve(pre.reduced, kind="restatement"))
    assert back.status_name == "OPTIMAL"
    assert rel(back.objective_value, want.objective_value) < 1e-9
    cert = verify_oracle.certificate(mdl, back.primal, back.dual_row, back.status, back.objective_value,
                                     back.duality_gap)
    assert cert["is_valid"] and cert["relative_gap"] < 1e-9 and cert["max_dual_infeasibility"] < 1e-9
    assert "Presolve removed" in back.message


def _tiny(rows, lb=None, ub=None, obj=(1.0, 1.0)):
    """Two columns; rows = list of (coefs (a0, a1), sense, rhs)."""
    cp, ri, va = [0], [], []
    for j in range(2):
        for i, (a, _, _) in enumerate(rows):
            if a[j] != 0:
                ri.append(i)
                va.append(float(a[j]))
        cp.append(len(ri))
    return P._lp(2, len(rows), np.array(cp, dtype=np.int32), np.array(ri, dtype=np.int32), np.array(va),
                 np.array(obj), np.array([r[2] for r in rows], dtype=float),
                 np.array([r[1] for r in rows], dtype=np.int8), "tiny", lb=lb, ub=ub)


def test_presolve_decides_without_a_solve():
    infeasible = _tiny([((1, 0), abi.LE, 1.0), ((1, 0), abi.GE, 2.0), ((1, 1), abi.LE, 9.0)])
    pre = Presolved(infeasible)
    assert pre.status == abi.INFEASIBLE and "Infeasible (presolve)" in pre.message
    unbounded = _tiny([((1, 0), abi.LE, 1.0)], obj=(1.0, -1.0))  # x1 in no row, cost falls, no upper bound
    assert Presolved(unbounded).status == abi.UNBOUNDED
    fixed = _tiny([((2, 0), abi.EQ, 3.0), ((0, 1), abi.GE, 0.5)], obj=(1.0, 4.0))
    pre = Presolved(fixed)
    assert pre.status == abi.OPTIMAL and pre.reduced.n == 0
    r = pre.postsolve(None)
    assert r.status_name == "OPTIMAL" and np.allclose(r.primal, [1.5, 0.5]) and abs(r.objective_value - 3.5) < 1e-12
    # the multipliers of the two removed rows price the objective: 2 y0 = 1, y1 = 4
    assert np.allclose(r.dual_row, [0.5, 4.0])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2])
def test_presolved_solve_on_gpu(seed):
    mdl = P.presolve_lp_example(60, 200, seed)
    want = oracle.solve(mdl, kind="reference")
    r = solve_presolved(mdl)
    assert r.status_name == "OPTIMAL", r.message
    assert "Presolve removed" in r.message and "Re-solved" not in r.message
    assert rel(r.objective_value, want.objective_value) < 1e-8
    cert = verify_solution(mdl, r)
    assert cert["is_valid"] and cert["relative_gap"] < 1e-7, cert


@pytest.mark.gpu
def test_presolve_claim_is_checked_on_gpu():
    # presolve proves infeasibility; the one-call solve then solves the original model itself, as the
    # reference's engine does, and says so
    infeasible = _tiny([((1, 0), abi.LE, 1.0), ((1, 0), abi.GE, 2.0), ((1, 1), abi.LE, 9.0)])
    r = solve_presolved(infeasible)
    assert "Re-solved without presolve because presolve reported infeasibility" in r.message
    assert r.status_name != "OPTIMAL"
