"""GPU QP parity: the convex-sequence (LISWET) shape against the reference's results, including
its published n = 20000 projection (golden vector from the reference's benchmark report), and QPs
whose Hessian couples variables (the reference's off-diagonal regression QP and its portfolio QP
with a diagonally dominant coupled covariance, test_correctness_regressions.cpp:263-330)."""
import json
import os

import numpy as np
import pytest

from sovereign_b200 import problems as P
from sovereign_b200.ipm import QpInteriorPointOptions, QpInteriorPointSolver

# The reference's answer on this shape comes from its exact active-set path (extended precision).
# The FP64 interior point stops at its 1e-8 gap; its objective then sits within a few 1e-8 of the
# exact optimum (measured: 1.6e-8 at n = 2002), the bar used here.
TIGHT = QpInteriorPointOptions(max_iterations=300)
OBJ_TOL = 5e-8

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
QP = json.load(open(os.path.join(GOLDEN, "qp_reference.json")))


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.mark.parametrize("key", ["convex_sequence_qp(52,3)", "convex_sequence_qp(202,3)", "convex_sequence_qp(2002,3)"])
def test_convex_sequence_matches_reference(key):
    g = QP[key]
    name, args = g["spec"]
    r = QpInteriorPointSolver(TIGHT).solve(getattr(P, name)(*args))
    assert r.status_name == "OPTIMAL", r.message
    assert rel(r.objective_value, g["objective"]) < OBJ_TOL


@pytest.mark.xfail(reason="FP64 normal equations of the n = 20000 convex-sequence QP have condition ~1e16; the "
                          "reference solves this shape in extended precision", strict=False)
def test_liswet_n20000_published_projection():
    g = np.load(os.path.join(GOLDEN, "liswet_n20000.npz"))
    mdl = P.convex_sequence_qp(len(g["c"]), 0, target=g["c"], with_constant=False)
    r = QpInteriorPointSolver(TIGHT).solve(mdl)
    assert r.status_name == "OPTIMAL", r.message
    assert rel(r.objective_value, float(g["objective"])) < OBJ_TOL
    assert np.max(np.abs(r.primal - g["x"])) < 1e-3
    # feasibility of the returned sequence: second differences >= 0
    assert np.min(r.primal[:-2] - 2 * r.primal[1:-1] + r.primal[2:]) > -1e-7


def test_default_options_stop_at_reference_tolerance():
    r = QpInteriorPointSolver().solve(P.convex_sequence_qp(202, 3))
    assert r.status_name == "OPTIMAL" and r.duality_gap < 1e-8
    assert rel(r.objective_value, QP["convex_sequence_qp(202,3)"]["objective"]) < 1e-7


def test_xspace_option_small_sequence_exact():
    # the x-space option eliminates the slacks; on a small instance it lands on the reference's
    # exact active-set objective
    from sovereign_b200 import abi
    from sovereign_b200.ipm import _solve
    o = QpInteriorPointOptions(max_iterations=300).to_abi(qp=True)
    o.factorization = abi.FACTOR_XSPACE
    rx = _solve(P.convex_sequence_qp(52, 3), o, True, False, False, None)
    assert rx.status_name == "OPTIMAL" and "x-space" in rx.message
    assert rel(rx.objective_value, QP["convex_sequence_qp(52,3)"]["objective"]) < 1e-8


# the reference's own bar between its dense and sparse KKT paths on the portfolio QP
# (test_correctness_regressions.cpp:318-320)
COUPLED_TOL = 1e-7


@pytest.mark.parametrize("key", ["small_qp_offdiagonal()", "reference_portfolio(60,5)", "reference_portfolio(300,12)"])
def test_coupled_hessian_matches_reference(key):
    g = QP[key]
    name, args = g["spec"]
    r = QpInteriorPointSolver().solve(getattr(P, name)(*args))
    assert r.status_name == "OPTIMAL", r.message
    assert "H = Q + X^-1 S dense" in r.message
    assert rel(r.objective_value, g["objective"]) < COUPLED_TOL
    assert np.all(np.abs(np.asarray(r.primal[:len(g["primal_head"])]) - np.asarray(g["primal_head"])) < 1e-6)


def test_coupled_hessian_known_answer():
    # QpAccuracy.OffDiagonalHessianTermsCountOnce: x = y = 0.4, objective -0.4
    r = QpInteriorPointSolver().solve(P.small_qp_offdiagonal())
    assert r.status_name == "OPTIMAL", r.message
    assert abs(r.primal[0] - 0.4) < 1e-7 and abs(r.primal[1] - 0.4) < 1e-7
    assert abs(r.objective_value + 0.4) < 1e-8


@pytest.mark.parametrize("key", ["reference_portfolio(60,5)@max8", "reference_portfolio(300,12)@max10",
                                 "reference_portfolio(60,5)@max5"])
def test_mehrotra_retry_matches_reference(key):
    # an iteration limit short enough to stop the default start: the reference then retries from
    # Mehrotra's starting point and reports both attempts' iterations (qp_interior_point.cpp:3166-3180)
    g = QP[key]
    name, args = g["spec"]
    r = QpInteriorPointSolver(QpInteriorPointOptions(max_iterations=g["max_iterations"])).solve(getattr(P, name)(*args))
    assert r.status_name == g["status"], r.message
    if g["status"] == "OPTIMAL":
        assert r.iterations > g["max_iterations"]  # the second attempt ran
        assert abs(r.iterations - g["iterations"]) <= 2
        assert rel(r.objective_value, g["objective"]) < COUPLED_TOL
    else:
        assert "| Mehrotra starting point:" in r.message
