"""GPU parity: the B200 engine against the reference's own results (golden vectors made by the
reference, tests/golden/make_golden.py) and against the oracle restatement on the same seeded
inputs. Objectives must match to 1e-8 relative, with residuals at the reference's tolerance."""
import json
import os

import numpy as np
import pytest

import oracle
from sovereign_b200 import abi, problems as P
from sovereign_b200.ipm import InteriorPointOptions, InteriorPointSolver, autotune, solve_batch

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
LP = json.load(open(os.path.join(GOLDEN, "lp_reference.json")))
SINGLE = [k for k, v in LP.items() if isinstance(v.get("spec"), list) and v["spec"][0] != "multicommodity"]
TOL = 1e-8  # relative objective tolerance


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def model_of(spec):
    name, args = spec
    if name == "multicommodity":
        return P.MulticommodityFamily().instance_from_seed(args[0])[0]
    return getattr(P, name)(*args)


@pytest.mark.parametrize("key", SINGLE + ["multicommodity(100)"])
def test_fp64_matches_reference(key):
    g = LP[key]
    r = InteriorPointSolver().solve(model_of(g["spec"]), with_diag=True)
    assert r.status_name == "OPTIMAL", r.message
    assert rel(r.objective_value, g["objective"]) < TOL
    assert r.primal_residual < 1e-9 and r.dual_residual < 1e-9 and r.duality_gap < 1e-9
    # same algorithm in FP64: never more iterations than the reference (dependent rows are dropped
    # exactly instead of being carried through a near-singular LU, which can cost it iterations)
    assert r.iterations <= g["iterations"] + 1
    assert "Normal equations" in r.message


@pytest.mark.parametrize("key", ["reference_staircase(8,40)", "transport(50,50,0)", "reference_transport(60)",
                                 "random_sparse_lp(100,500,8,1)", "bounded_lp_example()", "multicommodity(100)",
                                 "budget_lp(400,4000,6,7)", "budget_lp(2000,40000,6,3)"])
def test_sparse_factorization_matches_reference(key, monkeypatch):
    # the reference's sparse path (SOVEREIGN_IPM_NORMAL_EQUATIONS=sparse): minimum-degree order on the
    # host, numeric L D L' and its solves on the GPU level by level in the elimination tree
    monkeypatch.setenv("SOVEREIGN_IPM_NORMAL_EQUATIONS", "sparse")
    g = LP[key]
    r = InteriorPointSolver().solve(model_of(g["spec"]), with_diag=True)
    assert r.status_name == "OPTIMAL", r.message
    # a nearly dense normal matrix (2000 random rows over 40000 columns) is factored densely instead
    assert "sparse LDL^T on the GPU" in r.message or "the sparse factor would be nearly dense" in r.message
    assert rel(r.objective_value, g["objective"]) < TOL
    assert r.primal_residual < 1e-9 and r.dual_residual < 1e-9 and r.duality_gap < 1e-9
    assert r.iterations <= g["iterations"] + 1


@pytest.mark.parametrize("key", ["transport(50,50,0)", "random_sparse_lp(200,1000,8,2)", "reference_transport(40)",
                                 "multicommodity(101)"])
def test_mixed_precision_matches_reference(key):
    g = LP[key]
    opts = InteriorPointOptions(precision=abi.PRECISION_MIXED)
    r = InteriorPointSolver(opts).solve(model_of(g["spec"]), with_diag=True)
    assert r.status_name == "OPTIMAL", r.message
    assert rel(r.objective_value, g["objective"]) < TOL
    assert r.diagnostics["pcg_iterations"] > 0


def test_batch_matches_reference():
    g = LP["transport_batch"]
    models = P.transport_batch(**g["spec"])
    res = solve_batch(models)
    for k, r in enumerate(res):
        assert r.status_name == "OPTIMAL", (k, r.message)
        assert rel(r.objective_value, g["objectives"][k]) < TOL, k
        assert r.iterations <= g["iterations"][k] + 1, k


def test_batch_headline_all_4096_match_reference():
    # every LP of the 4096-LP batched workload against the reference. Where the reference's dense LU
    # stops short of OPTIMAL (a pivot under its 1e-14 floor on a dependent row), the golden holds
    # the objective of the reference's own sparse L D L' path, which drops the dependent row as the
    # GPU factorization does
    g = np.load(os.path.join(GOLDEN, "transport4096_reference.npz"))
    want = np.where(g["status"] == 0, g["objective"], g["sparse_objective"])
    assert np.all((g["status"] == 0) | (g["sparse_status"] == 0))
    res = solve_batch(P.transport_batch(4096, seed=2026), with_diag=False)
    errs = np.array([rel(r.objective_value, w) for r, w in zip(res, want)])
    assert all(r.status_name == "OPTIMAL" for r in res)
    assert errs.max() < TOL, (int(errs.argmax()), errs.max())
    assert max(max(r.primal_residual, r.dual_residual, r.duality_gap) for r in res) < 1e-9


def random_lp_family(count, seed):
    """Small random LPs whose rows share several columns (3-6 entries per column), so entries of the
    normal matrix receive several terms in the batched kernel's assembly."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        m = int(rng.integers(20, 121))
        out.append(P.random_sparse_lp(m, int(rng.integers(2 * m, 5 * m)), int(rng.integers(3, 7)), 5000 + k))
    return out


def test_batch_random_lps_match_reference():
    models = random_lp_family(48, 11)
    res = solve_batch(models)
    for k, (mdl, r) in enumerate(zip(models, res)):
        ref = oracle.solve(mdl, kind="reference")
        assert ref.status_name == "OPTIMAL", (k, ref.message)
        assert r.status_name == "OPTIMAL", (k, r.message)
        assert rel(r.objective_value, ref.objective_value) < TOL, (k, r.objective_value, ref.objective_value)
        assert r.iterations <= ref.iterations + 2, k


def test_batch_error_names_the_callers_model():
    # a call of 3072 LPs runs in pipelined parts; a model that cannot be built is named by its
    # position in the caller's list, not within its part
    import dataclasses
    models = P.transport_batch(3072, seed=41)
    bad = models[2900]
    ub = bad.ub.copy()
    ub[0] = -1.0  # below its lower bound 0
    models[2900] = dataclasses.replace(bad, ub=ub, _keep=[])
    with pytest.raises(Exception, match=r"model 2900: Inconsistent bounds"):
        solve_batch(models)


def test_batch_run_to_run():
    # transportation LPs: every normal-matrix entry receives one term, so two runs agree bit for bit;
    # random LPs (several terms per entry, summed by shared-memory atomics in arrival order) agree to
    # far below the 1e-8 parity tolerance (measured: 2.5e-11)
    t = P.transport_batch(256, seed=17)
    a, b = solve_batch(t), solve_batch(t)
    for x, y in zip(a, b):
        assert x.objective_value == y.objective_value and x.iterations == y.iterations
        np.testing.assert_array_equal(x.primal, y.primal)
    r = random_lp_family(32, 12)
    a, b = solve_batch(r), solve_batch(r)
    assert max(rel(x.objective_value, y.objective_value) for x, y in zip(a, b)) < 1e-9


@pytest.mark.parametrize("threads", ["128", "129", "256", "257", "512"])
def test_batch_every_cta_width(threads, monkeypatch):
    # the per-bucket kernel shape (width; odd codes: the register-capped lean variants) is a tuning
    # choice only: every shape gives the reference's answers
    monkeypatch.setenv("SOVEREIGN_BATCH_THREADS", threads)
    g = LP["transport_batch"]
    res = solve_batch(P.transport_batch(**g["spec"]))
    for k, r in enumerate(res):
        assert r.status_name == "OPTIMAL", (k, r.message)
        assert rel(r.objective_value, g["objectives"][k]) < TOL, k


def test_autotune_reports_every_bucket():
    models = P.transport_batch(64, seed=5)
    rep = json.loads(autotune(models))
    assert rep and all(set(v) >= {"128", "256", "512", "chosen", "count"} for v in rep.values())
    assert sum(v["count"] for v in rep.values()) == len(models)
    res = solve_batch(models)
    assert all(r.status_name == "OPTIMAL" for r in res)


def test_batch_mixed_sizes_and_fallback():
    # the batched kernel takes m <= 128; larger LPs in the same call go through the single engine
    models = [P.transport(50, 50, 0), P.reference_staircase(8, 40), P.transport(10, 10, 3), P.bounded_lp_example()]
    res = solve_batch(models)
    for mdl, r in zip(models, res):
        ref = oracle.solve(mdl, kind="restatement")
        assert r.status_name == "OPTIMAL" and rel(r.objective_value, ref.objective_value) < TOL


def test_batch_equals_single_engine_primal():
    models = P.transport_batch(8, seed=9)
    res = solve_batch(models)
    for mdl, r in zip(models, res):
        s = InteriorPointSolver().solve(mdl)
        assert rel(r.objective_value, s.objective_value) < 1e-10
        np.testing.assert_allclose(r.primal, s.primal, rtol=1e-6, atol=1e-6)


def with_explicit_zero(mdl):
    """The same LP with an explicit 0.0 entry in its first column: not a plain column layout, so the
    batch builds it on the host (build_std_form) instead of in place."""
    import dataclasses
    rows = set(mdl.row_idx[mdl.col_ptr[0]:mdl.col_ptr[1]].tolist())
    r = next(i for i in range(mdl.m) if i not in rows)
    e = int(mdl.col_ptr[0]) + int(np.searchsorted(mdl.row_idx[mdl.col_ptr[0]:mdl.col_ptr[1]], r))
    col_ptr = mdl.col_ptr.copy()
    col_ptr[1:] += 1
    return dataclasses.replace(mdl, col_ptr=col_ptr, row_idx=np.insert(mdl.row_idx, e, r).astype(np.int32),
                               values=np.insert(mdl.values, e, 0.0), name=mdl.name + "_zero", _keep=[])


def test_batch_device_scaling_matches_host_builder():
    # LPs built in place are scaled on the device (k_batch_scale) and their results unscaled there
    # (k_batch_publish); the single engine scales on the host. The arithmetic is the same, so the
    # coefficient range after scaling is equal bit for bit and the published solutions agree to the
    # engines' tolerance (row duals through A'y). Covers bounds (shift, UB rows), Le/Ge slacks, a
    # maximisation, an LP the batch scales on the host (explicit zero entry), scaling off, and the
    # IPM-space copies.
    models = [P.bounded_lp_example(), P.transport(12, 9, 2), with_explicit_zero(P.transport(8, 7, 1)),
              P.random_sparse_lp(40, 90, 3, 4)]
    for opts in (InteriorPointOptions(), InteriorPointOptions(enable_scaling=False)):
        res = solve_batch(models, opts, with_diag=True)
        res_ipm = solve_batch(models, opts, with_ipm=True)
        for k, (mdl, r, ri) in enumerate(zip(models, res, res_ipm)):
            s = InteriorPointSolver(opts).solve(mdl, with_diag=True)
            assert r.status_name == "OPTIMAL" and s.status_name == "OPTIMAL", (k, r.message)
            for key in ("scaling_applied", "coefficient_min_abs_before", "coefficient_max_abs_before",
                        "coefficient_min_abs_after", "coefficient_max_abs_after"):
                assert r.diagnostics[key] == s.diagnostics[key], (k, key)
            assert rel(r.objective_value, s.objective_value) < 1e-9, k
            np.testing.assert_allclose(r.primal, s.primal, rtol=1e-6, atol=1e-6)
            np.testing.assert_allclose(r.dual_col, s.dual_col, rtol=1e-5, atol=1e-6)
            # row duals are unique up to the null space of A' (a transportation LP's supply and demand
            # duals can shift by opposite constants): compare A' y
            A = mdl.dense_A()
            np.testing.assert_allclose(A.T @ r.dual_row, A.T @ s.dual_row, rtol=1e-5, atol=1e-5)
            # the with-iterates solve publishes the same values: bit for bit where every normal-matrix
            # entry gets one term (no two rows share more than one column); otherwise an entry sums
            # several terms by shared-memory atomics in arrival order, and two solves agree to rounding
            nz = (A != 0).astype(int)
            shared = nz @ nz.T
            np.fill_diagonal(shared, 0)
            if shared.max() > 1:
                np.testing.assert_allclose(ri.primal, r.primal, rtol=1e-9, atol=1e-12)
            else:
                np.testing.assert_array_equal(ri.primal, r.primal)
            assert np.all(np.isfinite(ri.ipm_x)) and np.any(ri.ipm_x != 0.0)


def test_result_contract_matches_restatement():
    mdl = P.bounded_lp_example()
    r = InteriorPointSolver().solve(mdl, with_diag=True)
    o = oracle.solve(mdl, kind="restatement", with_diag=True)
    assert r.status == o.status and rel(r.objective_value, o.objective_value) < TOL
    np.testing.assert_allclose(r.primal, o.primal, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(r.dual_row, o.dual_row, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(r.dual_col, o.dual_col, rtol=1e-5, atol=1e-6)
    assert r.diagnostics["scaling_applied"] and r.diagnostics["history_iterations"][:3] == [1, 2, 3]
    assert r.diagnostics["coefficient_max_abs_after"] == pytest.approx(o.diagnostics["coefficient_max_abs_after"])


def test_iteration_limit_returns_best_candidate():
    mdl = P.reference_transport(30)
    r = InteriorPointSolver(InteriorPointOptions(max_iterations=1, optimality_tol=1e-14)).solve(mdl)
    o = oracle.solve(mdl, kind="restatement", max_iterations=1)
    assert r.status == o.status and r.status_name in ("FEASIBLE", "NUMERICAL_ERROR")
    assert r.has_objective_value and "Optimality is not proven" in r.message
    assert rel(r.objective_value, o.objective_value) < 1e-6


def test_inconsistent_bounds_and_degenerate_models():
    bad = P.bounded_lp_example()
    bad.ub = bad.ub.copy()
    bad.ub[0] = 0.0
    r = InteriorPointSolver().solve(bad)
    assert r.status_name == "ERROR" and r.message.startswith("IPM error: Inconsistent bounds")
    # no constraints: x at its lower bounds (interior_point.cpp:464-478)
    free = P.bounded_lp_example()
    free.m = 0
    free.rhs = np.zeros(0)
    free.sense = np.zeros(0, dtype=np.int8)
    free.col_ptr = np.zeros(free.n + 1, dtype=np.int32)
    free.row_idx = np.zeros(0, dtype=np.int32)
    free.values = np.zeros(0)
    free.ub = np.full(free.n, 1e30)
    r = InteriorPointSolver().solve(free)
    assert r.status_name == "OPTIMAL" and r.message == "Optimal (no constraints) via IPM path."
    np.testing.assert_allclose(r.primal, free.lb)


def test_dependent_rows_are_dropped():
    # balanced transport has a redundant equality row: the normal matrix is singular
    from sovereign_b200.ipm import normal_factor_solve
    mdl = P.reference_transport(12)
    # with weights 100 the dependent direction's pivot (~1e-12 shift plus rounding) sits far below
    # the relative threshold 1e-13 * diag ~ 1.2e-10, so the rule must drop exactly one row
    d = np.full(mdl.n, 100.0)
    rhs = mdl.dense_A() @ np.random.default_rng(1).standard_normal(mdl.n)
    z, dropped = normal_factor_solve(mdl.m, mdl.n, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs)
    assert dropped == 1
    A = mdl.dense_A()
    Mm = A @ np.diag(d) @ A.T
    np.testing.assert_allclose(Mm @ z, rhs, rtol=1e-8, atol=1e-7 * np.abs(rhs).max())


def test_batch_per_lp_options():
    # option blocks one per LP (opt_stride): LP 0 gets a 3-iteration cap, the others the defaults
    from sovereign_b200 import _lib
    import ctypes as C
    models = P.transport_batch(6, seed=21)
    opts = (abi.SovOptions * len(models))(*[abi.default_options() for _ in models])
    opts[0].max_iterations = 3
    res = solve_batch_raw(models, opts, C.sizeof(abi.SovOptions))
    assert res[0].status_name in ("FEASIBLE", "NUMERICAL_ERROR") and res[0].iterations <= 3
    for r in res[1:]:
        assert r.status_name == "OPTIMAL"


def solve_batch_raw(models, opts, stride):
    import ctypes as C
    from sovereign_b200 import _lib
    from sovereign_b200.model import ResultBuffers
    bufs = [ResultBuffers(m) for m in models]
    arr = (abi.SovModel * len(models))(*[m.to_abi() for m in models])
    res = (abi.SovResult * len(models))(*[b.raw for b in bufs])
    _lib.check(_lib.load().sov_lp_solve_batch(len(models), arr, opts, stride, res))
    out = []
    for b, r in zip(bufs, res):
        b.raw = r
        out.append(b.to_result())
    return out


def test_batch_warm_start_saves_iterations():
    # start each LP of the batch from its own iterate at the start of iteration 6 (single engine):
    # the batched kernel takes it (safeguard passed), converges to the same optimum, in fewer steps
    models = P.transport_batch(24, seed=33)
    early = [InteriorPointSolver(InteriorPointOptions(ipm_iterate_at=6)).solve(m, with_ipm=True) for m in models]
    cold = solve_batch(models, with_diag=True)
    warm = solve_batch(models, warm_starts=[(e.ipm_x, e.ipm_y, e.ipm_s) for e in early], with_diag=True)
    for c, w in zip(cold, warm):
        assert c.status_name == "OPTIMAL" and w.status_name == "OPTIMAL"
        assert rel(w.objective_value, c.objective_value) < 1e-8
    assert sum(w.diagnostics["warm_start_used"] for w in warm) >= len(models) - 2
    assert not any(c.diagnostics["warm_start_used"] for c in cold)
    assert np.mean([w.iterations for w in warm]) <= np.mean([c.iterations for c in cold]) - 3


def test_large_network_takes_the_sparse_path():
    # a 130 x 130 grid min-cost flow: normal matrix of order 16900, past the dense factorization, so
    # AUTO takes the sparse L D L' (the reference: sparse LDL^T, nnz(L) = 409164)
    g = LP["grid_network_lp(130)"]
    r = InteriorPointSolver().solve(P.grid_network_lp(130))
    assert r.status_name == "OPTIMAL", r.message
    assert "sparse LDL^T on the GPU" in r.message
    assert rel(r.objective_value, g["objective"]) < TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config1_full_size_matches_reference(precision):
    # the random LP at its full size (m = 2000, n = 10000, 8 nonzeros per column), FP64 and mixed
    # precision (FP32 tensor-core Cholesky preconditioning FP64 PCG), against the reference's solution
    g = np.load(os.path.join(GOLDEN, "c1_reference.npz"))
    prec = abi.PRECISION_FP64 if precision == "fp64" else abi.PRECISION_MIXED
    r = InteriorPointSolver(InteriorPointOptions(precision=prec)).solve(P.random_sparse_lp(2000, 10000, 8, 1),
                                                                        with_diag=True)
    assert r.status_name == "OPTIMAL", r.message
    assert rel(r.objective_value, float(g["objective"])) < TOL
    assert r.primal_residual <= 1e-8 and r.dual_residual <= 1e-8 and r.duality_gap <= 1e-8
    assert r.iterations <= int(g["iterations"]) + 1
    # the optimum of a random LP is unique: the primal agrees with the reference's
    np.testing.assert_allclose(r.primal, g["primal"], rtol=0, atol=1e-6 * max(1.0, np.abs(g["primal"]).max()))
