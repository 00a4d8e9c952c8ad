"""GPU parity of the sparse quasi-definite KKT path, K = [Q + X^-1 S + delta I, A'; A, -delta I]
(qp_interior_point.cpp:415-655), against the reference's QpInteriorPointSolver on the same QPs:
Hessians that couple variables (the reference's off-diagonal regression QP, its portfolio QPs, a
tridiagonal-Hessian QP at n = 2000, 20000 and 200000, the last two beyond the dense-Hessian path)
and a free column without curvature. Golden values: tests/golden/make_golden.py (kkt section)."""
import json
import os

import numpy as np
import pytest

from sovereign_b200 import abi
from sovereign_b200 import problems as P
from sovereign_b200.ipm import QpInteriorPointOptions, _solve

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KKT = json.load(open(os.path.join(GOLDEN, "kkt_reference.json")))
QP = json.load(open(os.path.join(GOLDEN, "qp_reference.json")))
OBJ_TOL = 1e-8      # relative objective, the reference QP's optimality tolerance
PRIMAL_TOL = 1e-6   # strictly convex: the primal optimum is unique


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def solve(mdl, factorization=abi.FACTOR_AUTO, **kw):
    o = QpInteriorPointOptions(**kw).to_abi(qp=True)
    o.factorization = factorization
    return _solve(mdl, o, True, False, False, None)


@pytest.mark.parametrize("key", ["small_qp_offdiagonal()", "reference_portfolio(60,5)", "reference_portfolio(300,12)"])
def test_sparse_kkt_matches_reference_on_coupled_hessians(key):
    g = QP[key]
    name, args = g["spec"]
    r = solve(getattr(P, name)(*args), abi.FACTOR_SPARSE)
    assert r.status_name == "OPTIMAL", r.message
    assert "quasi-definite" in r.message
    assert rel(r.objective_value, g["objective"]) < OBJ_TOL
    assert np.max(np.abs(r.primal[:len(g["primal_head"])] - np.asarray(g["primal_head"]))) < PRIMAL_TOL


@pytest.mark.parametrize("key", list(KKT))
def test_kkt_path_matches_reference(key):
    # default options: the automatic choice takes the KKT system (a sparse coupled Hessian, or a
    # free column without curvature)
    g = KKT[key]
    name, args = g["spec"]
    r = solve(getattr(P, name)(*args))
    assert r.status_name == g["status"] == "OPTIMAL", r.message
    assert "quasi-definite" in r.message
    assert rel(r.objective_value, g["objective"]) < OBJ_TOL
    sample = r.primal[::g["primal_stride"]]
    assert np.max(np.abs(sample - np.asarray(g["primal_sample"]))) < PRIMAL_TOL
    assert r.primal_residual <= 1e-8 and r.dual_residual <= 1e-8 and r.duality_gap <= 1e-8
    assert abs(r.iterations - g["iterations"]) <= 3


def test_kkt_and_dense_hessian_paths_agree():
    # the same coupled QP through the dense H = Q + X^-1 S normal equations and through the KKT system
    mdl = P.coupled_chain_qp(2000, 1)
    rk = solve(mdl, abi.FACTOR_SPARSE)
    rd = solve(mdl, abi.FACTOR_DENSE)
    assert rk.status_name == rd.status_name == "OPTIMAL", (rk.message, rd.message)
    assert "quasi-definite" in rk.message and "H = Q + X^-1 S dense" in rd.message
    assert rel(rk.objective_value, rd.objective_value) < 1e-10
    assert np.max(np.abs(rk.primal - rd.primal)) < 1e-7


def test_kkt_run_to_run_identical():
    # the factor sums each destination's updates in a fixed order: bit-identical repeats
    mdl = P.coupled_chain_qp(2000, 1)
    a, b = solve(mdl), solve(mdl)
    assert a.iterations == b.iterations
    assert np.array_equal(a.primal, b.primal) and a.objective_value == b.objective_value


def test_free_column_without_curvature_requires_kkt():
    # the normal equations need H^-1: a dense factorization of them is refused for such a QP
    r = solve(P.free_intercept_qp(400, 12, 3), abi.FACTOR_DENSE)
    assert r.status_name == "ERROR" and "without curvature" in r.message
