"""GPU parity of the family path (sov_lp_solve_family): LPs that share A, bounds and senses solved
64 at a time with one symbolic analysis and interleaved vectors. Against the reference's answers on
the multicommodity instances of the golden set, and against the single-problem engine on families
larger than one launch (objectives, iterations, warm starts, captured iterates)."""
import json
import os

import numpy as np
import pytest

from sovereign_b200 import problems as P
from sovereign_b200._lib import SovError
from sovereign_b200.ipm import InteriorPointOptions, InteriorPointSolver, solve_family

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
LP = json.load(open(os.path.join(GOLDEN, "lp_reference.json")))
TOL = 1e-8


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def test_multicommodity_family_matches_reference():
    fam = P.MulticommodityFamily()
    keys = ["multicommodity(100)", "multicommodity(101)"]
    models = [fam.instance_from_seed(LP[k]["spec"][1][0])[0] for k in keys]
    res = solve_family(models, with_diag=True)
    for k, r in zip(keys, res):
        g = LP[k]
        assert r.status_name == "OPTIMAL", r.message
        assert "one symbolic factor for the family" in r.message
        assert rel(r.objective_value, g["objective"]) < TOL
        assert r.primal_residual < 1e-9 and r.dual_residual < 1e-9 and r.duality_gap < 1e-9
        assert abs(r.iterations - g["iterations"]) <= 1


def test_family_equals_single_engine_across_launches():
    # 70 instances: a full launch of 64 and one of 6
    fam = P.MulticommodityFamily()
    models = [fam.instance_from_seed(500 + k)[0] for k in range(70)]
    res = solve_family(models)
    single = [InteriorPointSolver().solve(m) for m in models[:: 7]]
    for k, s in zip(range(0, 70, 7), single):
        r = res[k]
        assert r.status_name == s.status_name == "OPTIMAL", (k, r.message)
        assert rel(r.objective_value, s.objective_value) < 1e-9, k
        assert abs(r.iterations - s.iterations) <= 1, (k, r.iterations, s.iterations)
    assert all(r.status_name == "OPTIMAL" for r in res)


def test_transport_family_matches_single_engine():
    fam = P.TransportFamily()
    models = [fam.instance_from_seed(k)[0] for k in range(40)]
    res = solve_family(models)
    for k in (0, 13, 39):
        s = InteriorPointSolver().solve(models[k])
        assert res[k].status_name == "OPTIMAL", res[k].message
        assert rel(res[k].objective_value, s.objective_value) < 1e-9
        assert np.max(np.abs(res[k].primal - s.primal)) < 1e-6 * max(1.0, np.max(np.abs(s.primal)))


def test_family_warm_starts_and_captured_iterates():
    # captured iterates at the start of iteration 6, fed back as warm starts: the safeguard keeps
    # them, the solves take fewer iterations and reach the same optima
    fam = P.MulticommodityFamily()
    models = [fam.instance_from_seed(700 + k)[0] for k in range(20)]
    cold = solve_family(models, InteriorPointOptions(ipm_iterate_at=6), with_ipm=True, with_diag=True)
    starts = [(r.ipm_x, r.ipm_y, r.ipm_s) for r in cold]
    warm = solve_family(models, warm_starts=starts, with_diag=True)
    for c, w in zip(cold, warm):
        assert c.status_name == w.status_name == "OPTIMAL", (c.message, w.message)
        assert rel(c.objective_value, w.objective_value) < 1e-8
        assert w.diagnostics["warm_start_used"] == 1
        assert w.iterations < c.iterations
    # the captured iterate equals the single engine's at the same iteration, to rounding
    s = InteriorPointSolver(InteriorPointOptions(ipm_iterate_at=6)).solve(models[3], with_ipm=True)
    assert np.max(np.abs(cold[3].ipm_x - s.ipm_x)) < 1e-6 * max(1.0, np.max(np.abs(s.ipm_x)))


def test_family_iteration_limit_and_structure_check():
    fam = P.MulticommodityFamily()
    models = [fam.instance_from_seed(900 + k)[0] for k in range(3)]
    res = solve_family(models, InteriorPointOptions(max_iterations=4))
    single = InteriorPointSolver(InteriorPointOptions(max_iterations=4)).solve(models[1])
    assert res[1].status_name == single.status_name
    assert "IPM stopped after 4 iterations" in res[1].message
    other = P.transport(10, 12, 0)
    with pytest.raises(SovError):
        solve_family([models[0], other])
