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

# The reference's answer on this shape comes from its structured paths in extended precision. The
# engine takes it through the x-space double-double path (separable Q, free variables, banded
# inequality rows) and meets the reference's objective to 1e-8 relative.
TIGHT = QpInteriorPointOptions(max_iterations=300)
OBJ_TOL = 1e-8

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


def test_liswet_n20000_published_projection():
    # the reference's published n = 20000 projection (its benchmark report), with the default
    # options (100 iterations), through the double-double x-space path
    g = np.load(os.path.join(GOLDEN, "liswet_n20000.npz"))
    mdl = P.convex_sequence_qp(len(g["c"]), 0, target=g["c"], with_constant=False)
    r = QpInteriorPointSolver().solve(mdl)
    assert r.status_name == "OPTIMAL", r.message
    assert "double-double" in r.message
    assert rel(r.objective_value, float(g["objective"])) < OBJ_TOL
    assert r.primal_residual <= 1e-8 and r.dual_residual <= 1e-8 and r.duality_gap <= 1e-8
    assert np.max(np.abs(r.primal - g["x"])) < 1e-5
    # feasibility of the returned sequence: second differences >= 0
    assert np.min(r.primal[:-2] - 2 * r.primal[1:-1] + r.primal[2:]) > -1e-9


def test_general_engine_remains_for_the_convex_sequence(monkeypatch):
    # SOVEREIGN_QP_DISABLE=xband sends the shape to the general engine (FP64 banded normal equations)
    monkeypatch.setenv("SOVEREIGN_QP_DISABLE", "xband")
    r = QpInteriorPointSolver(TIGHT).solve(P.convex_sequence_qp(202, 3))
    assert r.status_name == "OPTIMAL" and "double-double" not in r.message
    assert rel(r.objective_value, QP["convex_sequence_qp(202,3)"]["objective"]) < 1e-7


def test_default_options_stop_at_reference_tolerance():
    r = QpInteriorPointSolver().solve(P.convex_sequence_qp(202, 3))
    assert r.status_name == "OPTIMAL" and r.duality_gap < 1e-8
    assert rel(r.objective_value, QP["convex_sequence_qp(202,3)"]["objective"]) < OBJ_TOL
    # row duals: the multipliers of the >= rows, non-negative, zero on the rows that are slack
    assert np.min(r.dual_row) >= 0.0
    x = r.primal
    w = x[:-2] - 2 * x[1:-1] + x[2:]
    assert np.max(np.abs(w * r.dual_row)) < 1e-6


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


# coupled Hessians: the reference's objective to 1e-8 relative
COUPLED_TOL = 1e-8


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


def test_config2_full_size_matches_reference():
    # the convex-sequence QP at its full size (n = 20002, m = 20000, t = sin(4 pi i / n) + 0.1 N(0,1)).
    # The reference's structured path reaches the optimum but reports ERROR: its own certifier
    # measures a dual residual of 1.2e-7 against its 1e-8 bar. Its objective and primal are the
    # comparison; the engine must reach OPTIMAL at the reference QP's tolerances.
    g = np.load(os.path.join(GOLDEN, "c2_reference.npz"))
    r = QpInteriorPointSolver().solve(P.convex_sequence_qp(20002, 2))
    assert r.status_name == "OPTIMAL", r.message
    assert rel(r.objective_value, float(g["objective"])) < OBJ_TOL
    assert r.primal_residual <= 1e-8 and r.dual_residual <= 1e-8 and r.duality_gap <= 1e-8
    assert np.max(np.abs(r.primal - g["primal"])) < 1e-5
    assert np.min(r.primal[:-2] - 2 * r.primal[1:-1] + r.primal[2:]) > -1e-9


def test_partitioned_band_factor_equals_single_chain(monkeypatch):
    # the x-space path's factorization cut into segments (one per thread, separators last) against
    # the single chain over all columns (SOVEREIGN_XBAND_SEGMENTS=1): the same optimum
    mdl = P.convex_sequence_qp(4002, 5)
    part = QpInteriorPointSolver().solve(mdl)
    monkeypatch.setenv("SOVEREIGN_XBAND_SEGMENTS", "1")
    chain = QpInteriorPointSolver().solve(mdl)
    assert part.status_name == chain.status_name == "OPTIMAL", (part.message, chain.message)
    assert rel(part.objective_value, chain.objective_value) < 1e-12
    assert np.max(np.abs(part.primal - chain.primal)) < 1e-8
