"""Regenerate the golden fixtures under tests/golden/ from the reference itself.

Run in a checkout where the reference sources are available (oracle/Makefile builds
oracle/_ref/libsovref.so from them):

    python tests/golden/make_golden.py

    python tests/golden/make_golden.py headline c1   # only these sections

Writes
  lp_reference.json   InteriorPointSolver results (status, iterations, objective, gap, residuals,
                      primal checksum) on the seeded and regression LP models below, the LPs
                      with a dense budget row included
  transport4096_reference.npz
                      the reference's objective and status for every LP of the 4096-LP batched
                      workload (transport_batch(4096, seed=2026)); where its dense LU stops short of
                      OPTIMAL (a pivot under its 1e-14 floor), also the objective of its own sparse
                      L D L' path (SOVEREIGN_IPM_NORMAL_EQUATIONS=sparse), which drops dependent rows
  c1_reference.npz    the reference's solution of the random LP m=2000, n=10000, 8 nnz per column
                      (random_sparse_lp(2000, 10000, 8, 1)): objective, residuals, primal, row duals
                      (about ten minutes of CPU)
  c2_reference.npz    the reference's answer on the convex-sequence QP n=20002, m=20000
                      (convex_sequence_qp(20002, 2)): its structured LISWET path (Goldfarb-Idnani in
                      extended precision, about three minutes) returns the objective and primal but
                      status ERROR, because its certifier measures a dual residual of 1.2e-7
  qp_reference.json   QpInteriorPointSolver results on the QP models below
  kkt_reference.json  QpInteriorPointSolver results on QPs that take its sparse quasi-definite KKT
                      path (qp_interior_point.cpp:415-655): the tridiagonal-Hessian coupled_chain_qp
                      at n = 2000, 20000 and 200000 and the free-intercept regression QP (a free
                      column without curvature); objective, status, iterations, the primal's sum
                      and every KKT_STRIDE-th primal value
  liswet_n20000.npz   the reference's published LISWET projection at n = 20000
                      (benchmarks/reports/liswet_step6/n20000: input_c.txt, x.txt and the
                      objective printed in solver.stdout.json / independent.json)
Test code reads only these files; nothing at test time touches the reference tree.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from sovereign_b200 import problems as P  # noqa: E402

LISWET_DIR = os.path.join(oracle.REFERENCE_DIR, "benchmarks", "reports", "liswet_step6", "n20000")

LP_SPECS = [
    ("reference_transport", [20]), ("reference_transport", [40]), ("reference_transport", [60]),
    ("reference_staircase", [8, 40]), ("bounded_lp_example", []),
    ("transport", [50, 50, 0]), ("transport", [50, 50, 1]), ("transport", [50, 50, 2]),
    ("transport", [13, 37, 5]), ("transport", [60, 10, 7]),
    ("random_sparse_lp", [100, 500, 8, 1]), ("random_sparse_lp", [200, 1000, 8, 2]),
    ("random_sparse_lp", [500, 2500, 8, 1]), ("grid_network_lp", [130]),
]
DENSE_ROW_LP_SPECS = [("budget_lp", [400, 4000, 6, 7]), ("budget_lp", [2000, 40000, 6, 3])]
BATCH_SPEC = dict(count=64, seed=3)          # transport_batch sample of the 4096-LP workload
MULTICOMMODITY_SEEDS = [100, 101]            # MulticommodityFamily() instances
QP_SPECS = [("small_qp_offdiagonal", []), ("convex_sequence_qp", [52, 3]), ("convex_sequence_qp", [202, 3]),
            ("convex_sequence_qp", [2002, 3]), ("reference_portfolio", [300, 12]), ("reference_portfolio", [60, 5])]
KKT_SPECS = [("coupled_chain_qp", [2000, 1]), ("coupled_chain_qp", [20000, 2]), ("coupled_chain_qp", [200000, 5]),
             ("free_intercept_qp", [400, 12, 3]), ("free_intercept_qp", [2000, 30, 4])]
KKT_STRIDE = 97
QP_RETRY_SPECS = [("reference_portfolio", [60, 5], 8), ("reference_portfolio", [60, 5], 5),
                  ("reference_portfolio", [300, 12], 10)]


def build(name, args):
    return getattr(P, name)(*args)


def summarize(r, model=None):
    d = dict(status=r.status_name, iterations=r.iterations, objective=r.objective_value,
             duality_gap=r.duality_gap, primal_residual=r.primal_residual, dual_residual=r.dual_residual,
             message=r.message)
    if r.primal is not None:
        d["primal_sum"] = float(np.sum(r.primal))
        d["primal_head"] = [float(v) for v in r.primal[:8]]
    if r.dual_row is not None:
        d["dual_row_head"] = [float(v) for v in r.dual_row[:8]]
    return d


def headline():
    """Every LP of the 4096-LP batched workload through the reference (all host threads)."""
    models = P.transport_batch(4096, seed=2026)
    secs, obj, its, st = oracle.solve_many_reference(models)
    bad = np.flatnonzero(st != 0)
    sparse_obj = np.full(len(models), np.nan)
    sparse_st = np.full(len(models), -1, dtype=np.int32)
    os.environ["SOVEREIGN_IPM_NORMAL_EQUATIONS"] = "sparse"
    try:
        for i in bad:
            r = oracle.solve(models[i], kind="reference")
            sparse_obj[i], sparse_st[i] = r.objective_value, r.status
    finally:
        del os.environ["SOVEREIGN_IPM_NORMAL_EQUATIONS"]
    np.savez_compressed(os.path.join(HERE, "transport4096_reference.npz"), objective=obj, status=st, iterations=its,
                        sparse_objective=sparse_obj, sparse_status=sparse_st)
    print(f"headline: {len(models)} LPs in {secs:.1f} s, {len(bad)} not OPTIMAL on the dense path, "
          f"sparse path statuses {sparse_st[bad].tolist()}", flush=True)


def c1():
    """Config 1 at full size: random LP m=2000, n=10000, 8 nnz per column, seed 1."""
    mdl = P.random_sparse_lp(2000, 10000, 8, 1)
    r = oracle.solve(mdl, kind="reference")
    np.savez_compressed(os.path.join(HERE, "c1_reference.npz"), objective=r.objective_value, status=r.status,
                        iterations=r.iterations, duality_gap=r.duality_gap, primal_residual=r.primal_residual,
                        dual_residual=r.dual_residual, primal=r.primal, dual_row=r.dual_row,
                        seconds=r.solve_seconds, message=r.message)
    print("c1", r.status_name, r.iterations, r.objective_value, r.solve_seconds, flush=True)


def c2():
    """Config 2: the convex-sequence QP n=20002 (t = sin(4 pi i / n) + 0.1 N(0,1), seed 2)."""
    mdl = P.convex_sequence_qp(20002, 2)
    r = oracle.solve(mdl, qp=True, kind="reference")
    np.savez_compressed(os.path.join(HERE, "c2_reference.npz"), objective=r.objective_value, status=r.status,
                        primal=r.primal, seconds=r.solve_seconds, message=r.message[:300])
    print("c2", r.status_name, r.objective_value, r.solve_seconds, flush=True)


def dense_row_lps():
    """LPs with a dense budget row (rows longer than a warp's piece of work), added to
    lp_reference.json in place."""
    path = os.path.join(HERE, "lp_reference.json")
    with open(path) as f:
        lp = json.load(f)
    for name, args in DENSE_ROW_LP_SPECS:
        key = f"{name}({','.join(map(str, args))})"
        lp[key] = dict(spec=[name, args], **summarize(oracle.solve(build(name, args), kind="reference")))
        print("lp", key, lp[key]["status"], lp[key]["objective"], flush=True)
    with open(path, "w") as f:
        json.dump(lp, f, indent=1)


def kkt():
    """QPs on the reference's sparse quasi-definite KKT path."""
    out = {}
    for name, args in KKT_SPECS:
        mdl = build(name, args)
        r = oracle.solve(mdl, qp=True, kind="reference")
        key = f"{name}({','.join(map(str, args))})"
        d = summarize(r)
        d["seconds"] = r.solve_seconds
        d["primal_stride"] = KKT_STRIDE
        d["primal_sample"] = [float(v) for v in r.primal[::KKT_STRIDE]]
        out[key] = dict(spec=[name, args], **d)
        print("kkt", key, r.status_name, r.iterations, r.objective_value, flush=True)
    with open(os.path.join(HERE, "kkt_reference.json"), "w") as f:
        json.dump(out, f, indent=1)


def main(sections=()):
    oracle.build(reference=True)
    if "headline" in sections:
        headline()
    if "c1" in sections:
        c1()
    if "c2" in sections:
        c2()
    if "kkt" in sections:
        kkt()
    if "dense_row" in sections:
        dense_row_lps()
    if sections:
        return
    headline()
    lp = {}
    for name, args in LP_SPECS:
        mdl = build(name, args)
        lp[f"{name}({','.join(map(str, args))})"] = dict(spec=[name, args], **summarize(oracle.solve(mdl, kind="reference")))
        print("lp", name, args, lp[f"{name}({','.join(map(str, args))})"]["objective"], flush=True)
    batch = P.transport_batch(**BATCH_SPEC)
    lp["transport_batch"] = dict(spec=BATCH_SPEC, objectives=[], iterations=[], statuses=[])
    for mdl in batch:
        r = oracle.solve(mdl, kind="reference")
        lp["transport_batch"]["objectives"].append(r.objective_value)
        lp["transport_batch"]["iterations"].append(r.iterations)
        lp["transport_batch"]["statuses"].append(r.status_name)
    fam = P.MulticommodityFamily()
    for s in MULTICOMMODITY_SEEDS:
        mdl, _ = fam.instance_from_seed(s)
        lp[f"multicommodity({s})"] = dict(spec=["multicommodity", [s]], **summarize(oracle.solve(mdl, kind="reference")))
        print("mc", s, lp[f"multicommodity({s})"]["objective"], flush=True)
    with open(os.path.join(HERE, "lp_reference.json"), "w") as f:
        json.dump(lp, f, indent=1)
    dense_row_lps()

    qp = {}
    for name, args in QP_SPECS:
        mdl = build(name, args)
        key = f"{name}({','.join(map(str, args))})"
        qp[key] = dict(spec=[name, args], **summarize(oracle.solve(mdl, qp=True, kind="reference")))
        print("qp", key, qp[key]["objective"], flush=True)
    # the default start stopped by a short iteration limit, then the retry from Mehrotra's start
    for name, args, limit in QP_RETRY_SPECS:
        mdl = build(name, args)
        key = f"{name}({','.join(map(str, args))})@max{limit}"
        qp[key] = dict(spec=[name, args], max_iterations=limit,
                       **summarize(oracle.solve(mdl, qp=True, kind="reference", max_iterations=limit)))
        print("qp", key, qp[key]["status"], qp[key]["iterations"], flush=True)
    with open(os.path.join(HERE, "qp_reference.json"), "w") as f:
        json.dump(qp, f, indent=1)

    if os.path.isdir(LISWET_DIR):
        c = np.loadtxt(os.path.join(LISWET_DIR, "input_c.txt"))
        x = np.loadtxt(os.path.join(LISWET_DIR, "x.txt"))
        with open(os.path.join(LISWET_DIR, "independent.json")) as f:
            ind = json.load(f)
        obj = float(ind["independent"]["objective_qp"])
        np.savez_compressed(os.path.join(HERE, "liswet_n20000.npz"), c=c, x=x, objective=obj)
        print("liswet", len(c), obj)
    kkt()
    c1()
    c2()


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
