"""The oracle pinned: the C restatement against the reference's golden vectors and, where the
reference library was built, against the reference itself on the same inputs (CPU only)."""
import json
import os

import numpy as np
import pytest

import oracle
from sovereign_b200 import abi, problems as P

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
LP = json.load(open(os.path.join(GOLDEN, "lp_reference.json")))
QP = json.load(open(os.path.join(GOLDEN, "qp_reference.json")))
# the restatement factors M densely; above this size it is too slow for the CPU suite
SMALL_LP = [k for k, v in LP.items() if "spec" in v and isinstance(v["spec"], list)
            and v["spec"][0] not in ("multicommodity", "grid_network_lp")
            and k not in ("random_sparse_lp(500,2500,8,1)", "budget_lp(2000,40000,6,3)")]


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.mark.parametrize("key", SMALL_LP)
def test_restatement_matches_reference_golden(key):
    g = LP[key]
    name, args = g["spec"]
    r = oracle.solve(getattr(P, name)(*args), kind="restatement")
    assert r.status_name == g["status"]
    assert r.iterations == g["iterations"]
    # dense-path models are bit-identical; the staircase (reference: sparse LDL^T) agrees to rounding
    assert rel(r.objective_value, g["objective"]) < 1e-12
    assert abs(np.sum(r.primal) - g["primal_sum"]) <= 1e-9 * max(1.0, abs(g["primal_sum"]))


def test_restatement_matches_reference_golden_batch():
    g = LP["transport_batch"]
    models = P.transport_batch(**g["spec"])
    for k in range(0, len(models), 8):
        r = oracle.solve(models[k], kind="restatement")
        assert r.status_name == g["statuses"][k]
        assert r.iterations == g["iterations"][k]
        assert rel(r.objective_value, g["objectives"][k]) < 1e-12


@pytest.mark.parametrize("key", ["small_qp_offdiagonal()", "convex_sequence_qp(52,3)", "convex_sequence_qp(202,3)",
                                 "reference_portfolio(60,5)", "reference_portfolio(300,12)"])
def test_qp_restatement_matches_reference_golden(key):
    g = QP[key]
    name, args = g["spec"]
    r = oracle.solve(getattr(P, name)(*args), qp=True, kind="restatement")
    assert r.status_name == "OPTIMAL"
    # the reference takes its LISWET active-set path on the convex-sequence shape; the generic
    # interior point agrees to its 1e-8 tolerance
    exact = "offdiagonal" in key or "portfolio" in key  # same generic interior point as the reference
    assert rel(r.objective_value, g["objective"]) < (1e-12 if exact else 1e-8)


def test_qp_offdiagonal_known_answer():
    # QpAccuracy.OffDiagonalHessianTermsCountOnce: x = y = 0.4, objective -0.4
    r = oracle.solve(P.small_qp_offdiagonal(), qp=True, kind="restatement")
    assert abs(r.primal[0] - 0.4) < 1e-7 and abs(r.primal[1] - 0.4) < 1e-7
    assert abs(r.objective_value + 0.4) < 1e-8


@pytest.mark.skipif(not oracle.reference_available(), reason="reference library not built")
@pytest.mark.parametrize("seed", [11, 12, 13])
def test_restatement_matches_live_reference_random(seed):
    mdl = P.random_sparse_lp(60, 240, 6, seed)
    a = oracle.solve(mdl, kind="restatement", with_diag=True)
    b = oracle.solve(mdl, kind="reference", with_diag=True)
    assert a.status == b.status and a.iterations == b.iterations
    assert rel(a.objective_value, b.objective_value) < 1e-12
    np.testing.assert_allclose(a.primal, b.primal, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(a.dual_row, b.dual_row, rtol=1e-9, atol=1e-9)
    assert a.diagnostics["gap_history"] == pytest.approx(b.diagnostics["gap_history"], rel=1e-9, abs=1e-15)
    assert a.diagnostics["coefficient_max_abs_after"] == pytest.approx(b.diagnostics["coefficient_max_abs_after"])


@pytest.mark.skipif(not oracle.reference_available(), reason="reference library not built")
def test_restatement_failure_paths_match_reference():
    mdl = P.reference_transport(30)
    for kind in ("restatement", "reference"):
        r = oracle.solve(mdl, kind=kind, max_iterations=1)
        assert r.status_name in ("FEASIBLE", "NUMERICAL_ERROR")
        assert r.has_objective_value and "Optimality is not proven" in r.message
    a = oracle.solve(mdl, kind="restatement", max_iterations=1)
    b = oracle.solve(mdl, kind="reference", max_iterations=1)
    assert a.status == b.status and a.iterations == b.iterations
    assert rel(a.objective_value, b.objective_value) < 1e-12
    bad = P.bounded_lp_example()
    bad.ub = bad.ub.copy()
    bad.ub[0] = 0.0  # below lb = 1
    for kind in ("restatement", "reference"):
        r = oracle.solve(bad, kind=kind)
        assert r.status_name == "ERROR" and "Inconsistent bounds" in r.message


def test_oracle_spmv_and_normal_solve_against_numpy():
    mdl = P.random_sparse_lp(90, 130, 5, 7)
    A = mdl.dense_A()
    x = np.random.default_rng(0).standard_normal(130)
    y = np.random.default_rng(1).standard_normal(90)
    csc = (90, 130, mdl.col_ptr, mdl.row_idx, mdl.values)
    np.testing.assert_allclose(oracle.spmv(csc, x), A @ x, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(oracle.spmv(csc, y, transpose=True), A.T @ y, rtol=1e-12, atol=1e-12)
    d = np.random.default_rng(2).uniform(1e-3, 1e3, 130)
    rhs = np.random.default_rng(3).standard_normal(90)
    rc, z = oracle.normal_factor_solve(90, 130, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs)
    assert rc == 0
    Mm = A @ np.diag(d) @ A.T + 1e-12 * np.eye(90)
    np.testing.assert_allclose(Mm @ z, rhs, rtol=1e-8, atol=1e-8)


def test_ipm_form_scaling_and_slacks():
    f = oracle.ipm_form(P.bounded_lp_example())
    # 3 rows + 2 upper-bound rows; slacks for Le, Ge and both bound rows
    assert f["m"] == 5 and f["n"] == 3 + 4
    # after two passes of 1/sqrt(max) scaling every row and column max is close to 1
    A = np.zeros((f["m"], f["n"]))
    for j in range(f["n"]):
        for k in range(f["col_ptr"][j], f["col_ptr"][j + 1]):
            A[f["row_idx"][k], j] = f["values"][k]
    assert np.all(np.abs(A).max(axis=1) > 0.5) and np.all(np.abs(A).max(axis=0) > 0.5)
    np.testing.assert_allclose(f["shift"], [1.0, 0.0, 0.5])


def test_mlp_oracle_gradient_matches_finite_differences():
    from oracle import mlp_oracle
    dims = [5, 7, 7, 4]
    rng = np.random.default_rng(0)
    n = sum(dims[l + 1] * dims[l] + dims[l + 1] for l in range(3))
    p = rng.standard_normal(n) * 0.5
    x, t = rng.standard_normal((6, 5)), rng.standard_normal((6, 4))
    _, g, _ = mlp_oracle.loss_and_grad(p, dims, x, t)
    fd = np.zeros(n)
    for i in range(n):
        q = p.copy()
        q[i] += 1e-6
        a = mlp_oracle.loss_and_grad(q, dims, x, t)[0]
        q[i] -= 2e-6
        fd[i] = (a - mlp_oracle.loss_and_grad(q, dims, x, t)[0]) / 2e-6
    np.testing.assert_allclose(g, fd, atol=1e-7)
