"""CSC-native ingest of the reference's JSON model format (sov_model_from_json).

* CPU: oracle/_ref/json_check (tests/json_check.cpp) compares the ingest with the reference's own
  reader plus the IPM's index conversion, bit for bit, on the reference's transport datasets and on
  generated edge cases, and times both; the Python binding round-trips generated models.
* GPU: a model read from JSON solves to the same answer as the same model built in memory."""
import glob
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from sovereign_b200 import abi, problems as P
from sovereign_b200.ipm import InteriorPointSolver, load_model_json

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JSON_CHECK = os.path.join(ROOT, "oracle", "_ref", "json_check")
DATASETS = sorted(glob.glob(os.path.join(oracle.REFERENCE_DIR, "benchmarks", "datasets", "scale", "transport_*.json")))

SENSES = {abi.LE: "<=", abi.GE: ">=", abi.EQ: "="}


def to_json(mdl, names=None) -> str:
    """The reference's JSON format for a Model (model_to_json, json_io.cpp:86-108)."""
    names = names or [f"x{j}" for j in range(mdl.n)]
    rows = [dict(name=f"r{i}", sense=SENSES[int(mdl.sense[i])], rhs=float(mdl.rhs[i]), linear={})
            for i in range(mdl.m)]
    for j in range(mdl.n):
        for k in range(mdl.col_ptr[j], mdl.col_ptr[j + 1]):
            rows[mdl.row_idx[k]]["linear"][names[j]] = float(mdl.values[k])
    obj = dict(constant=float(mdl.obj_constant), linear={names[j]: float(mdl.obj[j]) for j in range(mdl.n)})
    if mdl.q_col_ptr is not None:
        q = {}
        for j in range(mdl.n):
            for k in range(mdl.q_col_ptr[j], mdl.q_col_ptr[j + 1]):
                q.setdefault(names[mdl.q_row_idx[k]], {})[names[j]] = float(mdl.q_values[k])
        obj["quadratic"] = q
    return json.dumps(dict(problem_type="QP" if mdl.is_qp else "LP", sense="maximize" if mdl.maximize else "minimize",
                           variables=[dict(name=names[j], type="continuous", lower_bound=float(mdl.lb[j]),
                                           upper_bound=float(mdl.ub[j])) for j in range(mdl.n)],
                           objective=obj, constraints=rows))


@pytest.mark.skipif(not os.path.exists(JSON_CHECK), reason="json_check is built with the reference library")
def test_ingest_matches_reference_reader():
    r = subprocess.run([JSON_CHECK] + DATASETS, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "failures 0" in r.stdout, r.stdout + r.stderr
    print(r.stdout.strip().splitlines()[-2])


@pytest.mark.parametrize("mdl", [P.transport(7, 9, 1), P.bounded_lp_example(), P.random_sparse_lp(30, 80, 4, 2),
                                 P.reference_portfolio(60, 5)], ids=["transport", "bounded", "random", "portfolio"])
def test_python_round_trip(mdl):
    got, names, rows = load_model_json(to_json(mdl))
    assert (got.n, got.m, got.maximize, got.obj_constant) == (mdl.n, mdl.m, mdl.maximize, mdl.obj_constant)
    for key in ("col_ptr", "row_idx", "values", "obj", "rhs", "sense", "lb", "ub"):
        np.testing.assert_array_equal(getattr(got, key), getattr(mdl, key), err_msg=key)
    assert names == [f"x{j}" for j in range(mdl.n)] and rows == [f"r{i}" for i in range(mdl.m)]
    assert (got.q_col_ptr is None) == (mdl.q_col_ptr is None)


def test_ingest_errors():
    from sovereign_b200._lib import SovError
    with pytest.raises(SovError, match="Unknown variable in constraint: zz"):
        load_model_json('{"problem_type": "LP", "variables": [{"name": "a"}], '
                        '"constraints": [{"sense": "<=", "rhs": 1, "linear": {"zz": 1}}]}')
    with pytest.raises(SovError, match="at byte"):
        load_model_json('{"problem_type": "LP", "variables": [{"name": "a"}')
    with pytest.raises(SovError, match="Unknown constraint sense"):
        load_model_json('{"problem_type": "LP", "variables": [], "constraints": [{"sense": "<", "rhs": 1}]}')


@pytest.mark.gpu
def test_json_model_solves_like_the_in_memory_model():
    mdl = P.random_sparse_lp(120, 400, 5, 6)
    got, _, _ = load_model_json(to_json(mdl))
    a, b = InteriorPointSolver().solve(mdl), InteriorPointSolver().solve(got)
    assert a.status_name == b.status_name == "OPTIMAL"
    assert a.objective_value == b.objective_value and a.iterations == b.iterations
    np.testing.assert_array_equal(a.primal, b.primal)
