"""The GPU certificate of an answer (sov_verify_solution) against the CPU restatement of
SolutionVerifier::verify and of the dual figures (oracle/verify_oracle.py): every figure to 1e-12,
the same verdict; an interior-point answer passes the verifier's checks at its default 1e-6 and
carries a dual certificate (reduced-cost signs and dual objective) that closes the gap; perturbed
answers fail with the right issue bits."""
import dataclasses

import numpy as np
import pytest

from oracle import verify_oracle
from sovereign_b200 import problems as P
from sovereign_b200.ipm import InteriorPointSolver, QpInteriorPointSolver, verify_solution

pytestmark = pytest.mark.gpu

KEYS = ("max_bound_violation", "max_constraint_violation", "recomputed_objective", "dual_objective",
        "max_dual_infeasibility", "relative_gap")


def _maximized(mdl):
    return dataclasses.replace(mdl, obj=-mdl.obj, maximize=True, _keep=[])


def _cases():
    return [("transport", P.transport(20, 30, 4), False), ("bounded", P.bounded_lp_example(), False),
            ("staircase", P.reference_staircase(8, 40), False), ("random", P.random_sparse_lp(80, 300, 5, 3), False),
            ("maximize", _maximized(P.transport(12, 9, 2)), False), ("portfolio", P.reference_portfolio(60, 5), True),
            ("convex_sequence", P.convex_sequence_qp(202, 3), True)]


def _close(got, want):
    for k in KEYS:
        assert abs(got[k] - want[k]) <= 1e-12 * max(1.0, abs(want[k])), (k, got[k], want[k])
    assert got["issues"] == want["issues"] and got["is_valid"] == want["is_valid"]


@pytest.mark.parametrize("name,mdl,qp", _cases(), ids=[c[0] for c in _cases()])
def test_certificate_of_ipm_answers(name, mdl, qp):
    r = (QpInteriorPointSolver() if qp else InteriorPointSolver()).solve(mdl)
    assert r.status_name == "OPTIMAL", r.message
    got = verify_solution(mdl, r)
    want = verify_oracle.certificate(mdl, r.primal, r.dual_row, r.status, r.objective_value, r.duality_gap)
    _close(got, want)
    # the verifier accepts the interior point as it is, and its duals close the gap
    assert got["is_valid"], got["issue_names"]
    assert got["relative_gap"] < 1e-7
    assert got["max_dual_infeasibility"] < 1e-6 * max(1.0, float(np.abs(mdl.obj).max()))


def test_certificate_flags_perturbed_answers():
    mdl = P.transport(15, 15, 7)
    r = InteriorPointSolver().solve(mdl)
    bad = dataclasses.replace(r, primal=r.primal.copy())
    bad.primal[3] = -1e-3                       # below its lower bound 0, and rows off by 1e-3
    got = verify_solution(mdl, bad)
    want = verify_oracle.certificate(mdl, bad.primal, bad.dual_row, bad.status, bad.objective_value, bad.duality_gap)
    _close(got, want)
    assert not got["is_valid"] and "bound" in got["issue_names"] and "constraint" in got["issue_names"]
    wrong = dataclasses.replace(r, objective_value=r.objective_value + 1.0)
    assert "objective" in verify_solution(mdl, wrong)["issue_names"]
    limit = dataclasses.replace(r, status=5)  # ITERATION_LIMIT: no feasible claim to check
    assert verify_solution(mdl, limit)["issue_names"] == ["no feasible status"]
