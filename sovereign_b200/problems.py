"""Seeded instance generators.

Workloads (all FP64, generated with numpy's PCG64 from an explicit seed, so the GPU engine and
the CPU oracles always see the same arrays):

* ``transport``            balanced transportation LP, ns sources x nt sinks (2-nnz columns of
                           ones, all rows equalities; one row is redundant). 50 x 50 is the
                           2500-variable single-LP workload; sizes drawn from U{10..60} make the
                           4096-LP batched workload.
* ``random_sparse_lp``     m x n with exactly k nonzeros N(0,1) per column at distinct uniform
                           rows; b = A x0, c = A'y0 + s0, feasible and bounded by construction.
* ``convex_sequence_qp``   min 1/2||x - t||^2 s.t. x_r - 2 x_{r+1} + x_{r+2} >= 0, free x
                           (the LISWET shape), t_i = sin(4 pi i / n) + 0.1 N(0,1).
* ``multicommodity``       a fixed random graph with arc capacities and costs, K commodities,
                           coupling (capacity) rows plus per-commodity conservation rows; each
                           instance perturbs demands and costs.
* ``wide_lp``              an LP far wider than L2 (m = 2000, n = 2M, 8 nnz per column) for the
                           HBM-bound passes of the single-problem engine.
* ``budget_lp``            random_sparse_lp plus one dense budget row over all columns.
* ``coupled_chain_qp``     min sum_i w_i/2 (x_{i+1} - x_i)^2 + sum_i d_i/2 x_i^2 - t'x over
                           0 <= x <= 2, a covering row per block of columns and one budget row:
                           a Hessian that couples neighbours (tridiagonal), the sparse coupled
                           shape that the quasi-definite KKT system takes at any size.
* ``free_intercept_qp``    ridge regression with a free, unpenalised intercept and box-bounded
                           coefficients: a free column without curvature.
* ``reference_transport`` / ``reference_staircase`` / ``reference_portfolio``: the deterministic
                           models of the reference's own regression tests
                           (tests/unit/test_correctness_regressions.cpp:74-111,157-180,263-290).
"""
from __future__ import annotations

import numpy as np

from .abi import EQ, GE, LE
from .model import Model

INF = 1e30


def _csc_from_triplets(n: int, cols: np.ndarray, rows: np.ndarray, vals: np.ndarray):
    order = np.lexsort((rows, cols))
    cols, rows, vals = cols[order], rows[order], vals[order]
    col_ptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(col_ptr, cols + 1, 1)
    col_ptr = np.cumsum(col_ptr).astype(np.int32)
    return col_ptr, rows.astype(np.int32), vals.astype(np.float64)


def _lp(n, m, col_ptr, row_idx, values, obj, rhs, sense, name, lb=None, ub=None, constant=0.0) -> Model:
    return Model(n=n, m=m, col_ptr=col_ptr, row_idx=row_idx, values=values,
                 obj=np.ascontiguousarray(obj, dtype=np.float64),
                 rhs=np.ascontiguousarray(rhs, dtype=np.float64),
                 sense=np.ascontiguousarray(sense, dtype=np.int8),
                 lb=np.zeros(n) if lb is None else np.ascontiguousarray(lb, dtype=np.float64),
                 ub=np.full(n, INF) if ub is None else np.ascontiguousarray(ub, dtype=np.float64),
                 obj_constant=constant, name=name)


def transport_structure(ns: int, nt: int, cost: np.ndarray, supply: np.ndarray, demand: np.ndarray,
                        name: str) -> Model:
    """x_ij (i-major), supply rows 0..ns-1 (sum_j x_ij = s_i), demand rows ns..ns+nt-1."""
    n = ns * nt
    i = np.repeat(np.arange(ns), nt)
    j = np.tile(np.arange(nt), ns)
    col_ptr = np.arange(0, 2 * n + 1, 2, dtype=np.int32)
    row_idx = np.empty(2 * n, dtype=np.int32)
    row_idx[0::2] = i
    row_idx[1::2] = ns + j
    values = np.ones(2 * n)
    rhs = np.concatenate([supply, demand]).astype(np.float64)
    return _lp(n, ns + nt, col_ptr, row_idx, values, cost.reshape(-1), rhs,
               np.full(ns + nt, EQ, dtype=np.int8), name)


def transport(ns: int, nt: int, seed: int) -> Model:
    """Costs U[1,100]; supplies U{10..100}; demands U{10..100} rescaled to integers with
    sum(demand) == sum(supply), the remainder going to the last sink."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cost = rng.uniform(1.0, 100.0, size=(ns, nt))
    supply = rng.integers(10, 101, size=ns).astype(np.float64)
    raw = rng.integers(10, 101, size=nt).astype(np.float64)
    total = supply.sum()
    demand = np.floor(raw * total / raw.sum())
    demand[-1] += total - demand.sum()
    return transport_structure(ns, nt, cost, supply, demand, f"transport_{ns}x{nt}_s{seed}")


def transport_batch(count: int, seed: int, lo: int = 10, hi: int = 60) -> list[Model]:
    """count transport LPs with ns, nt ~ U{lo..hi}; instance k uses seed * 1_000_003 + k."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = rng.integers(lo, hi + 1, size=(count, 2))
    return [transport(int(a), int(b), seed * 1_000_003 + k) for k, (a, b) in enumerate(sizes)]


def grid_network_lp(g: int) -> Model:
    """Min-cost flow on a g x g grid: both directions of every edge an arc (cost 1..10 by a fixed
    rule), 5 units from the corner node 0 to the opposite corner, conservation rows (all Eq). The
    normal matrix is the grid Laplacian: order g^2, sparse after a minimum-degree order."""
    m = g * g
    rows, vals, cost = [], [], []
    for i in range(g):
        for j in range(g):
            a = i * g + j
            for di, dj in ((1, 0), (0, 1)):
                ni, nj = i + di, j + dj
                if ni >= g or nj >= g:
                    continue
                b = ni * g + nj
                for d in (0, 1):
                    frm, to = (b, a) if d else (a, b)
                    r0, r1 = min(frm, to), max(frm, to)
                    rows += [r0, r1]
                    vals += [-1.0 if r0 == frm else 1.0, -1.0 if r1 == frm else 1.0]
                    cost.append(1.0 + ((a * 7 + b * 3 + d) % 10))
    n = len(cost)
    col_ptr = np.arange(0, 2 * n + 1, 2, dtype=np.int32)
    rhs = np.zeros(m)
    rhs[0], rhs[m - 1] = -5.0, 5.0
    return _lp(n, m, col_ptr, np.array(rows, dtype=np.int32), np.array(vals), np.array(cost), rhs,
               np.full(m, EQ, dtype=np.int8), f"grid_network_{g}x{g}")


def random_sparse_lp(m: int, n: int, k: int, seed: int) -> Model:
    rng = np.random.Generator(np.random.PCG64(seed))
    rows = np.argsort(rng.random((n, m)), axis=1)[:, :k] if m <= 4096 else \
        np.stack([rng.choice(m, size=k, replace=False) for _ in range(n)])
    rows = np.sort(rows, axis=1).astype(np.int32)
    vals = rng.standard_normal((n, k))
    col_ptr = np.arange(0, n * k + 1, k, dtype=np.int32)
    row_idx = np.ascontiguousarray(rows.reshape(-1))
    values = np.ascontiguousarray(vals.reshape(-1))
    x0 = rng.uniform(0.1, 1.0, size=n)
    y0 = rng.standard_normal(m)
    s0 = rng.uniform(0.1, 1.0, size=n)
    b = np.zeros(m)
    np.add.at(b, row_idx, values * np.repeat(x0, k))
    aty = (values * y0[row_idx]).reshape(n, k).sum(axis=1)
    c = aty + s0
    return _lp(n, m, col_ptr, row_idx, values, c, b, np.full(m, EQ, dtype=np.int8),
               f"random_sparse_{m}x{n}_k{k}_s{seed}")


def convex_sequence_qp(n: int, seed: int, target: np.ndarray | None = None,
                       with_constant: bool = True) -> Model:
    """min 1/2||x - t||^2 over free x with (1,-2,1) x >= 0 on every window of 3 (m = n - 2)."""
    m = n - 2
    if target is None:
        rng = np.random.Generator(np.random.PCG64(seed))
        i = np.arange(n)
        target = np.sin(4.0 * np.pi * i / n) + 0.1 * rng.standard_normal(n)
    t = np.ascontiguousarray(target, dtype=np.float64)
    r = np.arange(m)
    cols = np.concatenate([r, r + 1, r + 2])
    rows = np.concatenate([r, r, r])
    vals = np.concatenate([np.ones(m), -2.0 * np.ones(m), np.ones(m)])
    col_ptr, row_idx, values = _csc_from_triplets(n, cols, rows, vals)
    mdl = _lp(n, m, col_ptr, row_idx, values, -t, np.zeros(m), np.full(m, GE, dtype=np.int8),
              f"convex_sequence_{n}_s{seed}", lb=np.full(n, -INF), ub=np.full(n, INF),
              constant=0.5 * float(t @ t) if with_constant else 0.0)
    mdl.q_col_ptr = np.arange(n + 1, dtype=np.int32)
    mdl.q_row_idx = np.arange(n, dtype=np.int32)
    mdl.q_values = np.ones(n)
    return mdl


def wide_lp(m: int, n: int, k: int, seed: int) -> Model:
    """An LP far wider than L2: n columns of k entries N(0,1), one in each of k bands of m/k rows
    (rows sorted within a column), equality rows b = A x0, c = A'y0 + s0 (feasible, bounded). At
    m = 2000, n = 2M, k = 8: 16M nonzeros, each pass over A streams ~200 MB from HBM."""
    rng = np.random.default_rng(seed)
    band = m // k
    rows = (rng.integers(0, band, size=(n, k)) + np.arange(k)[None, :] * band).astype(np.int32)
    vals = rng.standard_normal((n, k))
    x0 = rng.uniform(0.1, 1.0, n)
    y0 = rng.standard_normal(m)
    s0 = rng.uniform(0.1, 1.0, n)
    row_idx = np.ascontiguousarray(rows.reshape(-1))
    values = np.ascontiguousarray(vals.reshape(-1))
    col_ptr = np.arange(0, n * k + 1, k, dtype=np.int32)
    b = np.bincount(row_idx, weights=values * np.repeat(x0, k), minlength=m)
    c = (values * y0[row_idx]).reshape(n, k).sum(axis=1) + s0
    return _lp(n, m, col_ptr, row_idx, values, c, b, np.full(m, EQ, dtype=np.int8), f"wide_lp_{m}x{n}")


def budget_lp(m: int, n: int, k: int, seed: int, fraction: float = 0.2) -> Model:
    """random_sparse_lp(m, n, k, seed) plus one dense row: sum_j x_j <= fraction * sum_j x0_j over
    all n columns (x0 the point the equalities were built from), a budget row longer than a warp's
    piece of work. Dual feasible (y0 with a zero budget multiplier), so bounded."""
    base = random_sparse_lp(m, n, k, seed)
    rng = np.random.Generator(np.random.PCG64(seed))
    rng.random((n, m)) if m <= 4096 else None  # the draws random_sparse_lp made, in order
    rng.standard_normal((n, k))
    x0 = rng.uniform(0.1, 1.0, size=n)
    cols = np.repeat(np.arange(n), k)
    rows = base.row_idx.astype(np.int64)
    vals = base.values
    cols = np.concatenate([cols, np.arange(n)])
    rows = np.concatenate([rows, np.full(n, m)])
    vals = np.concatenate([vals, np.ones(n)])
    col_ptr, row_idx, values = _csc_from_triplets(n, cols, rows, vals)
    rhs = np.concatenate([base.rhs, [fraction * float(np.sum(x0))]])
    sense = np.concatenate([base.sense, np.array([LE], dtype=np.int8)])
    return _lp(n, m + 1, col_ptr, row_idx, values, base.obj, rhs, sense, f"budget_lp_{m}x{n}")


def presolve_lp_example(m: int, n: int, seed: int) -> Model:
    """A random feasible, bounded LP (random_sparse_lp's construction, k = 4) with what presolve
    removes added: fixed columns (lb = ub = x0_j), singleton rows of every sense satisfied by x0
    (x_j <= x0_j + 0.3, -2 x_j >= -2 (x0_j + 0.4), x_j >= x0_j / 2, 3 x_j = 3 x0_j), an empty row
    (0 <= 5) and an empty column with a positive cost; some columns carry finite upper bounds."""
    base = random_sparse_lp(m, n, 4, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    # x0 of random_sparse_lp: redraw its stream up to the point where it draws x0
    r2 = np.random.Generator(np.random.PCG64(seed))
    np.argsort(r2.random((n, m)), axis=1)
    r2.standard_normal((n, 4))
    x0 = r2.uniform(0.1, 1.0, size=n)
    cols = [list(zip(base.row_idx[base.col_ptr[j]:base.col_ptr[j + 1]].tolist(),
                     base.values[base.col_ptr[j]:base.col_ptr[j + 1]].tolist())) for j in range(n)]
    rhs, sense = list(base.rhs), list(base.sense)
    picks = rng.choice(n, size=min(n, 24), replace=False)
    lb, ub = np.zeros(n + 1), np.full(n + 1, INF)
    for q, j in enumerate(picks):
        kind = q % 6
        if kind == 0:  # fixed column
            lb[j] = ub[j] = x0[j]
            continue
        if kind == 5:  # a finite upper bound
            ub[j] = x0[j] + 0.25
            continue
        row = len(rhs)
        a, b, s = [(1.0, x0[j] + 0.3, LE), (-2.0, -2.0 * (x0[j] + 0.4), GE), (1.0, 0.5 * x0[j], GE),
                   (3.0, 3.0 * x0[j], EQ)][kind - 1]
        cols[j].append((row, a))
        rhs.append(b)
        sense.append(s)
    rhs.append(5.0)  # an empty row
    sense.append(LE)
    cols.append([])  # an empty column, positive cost
    m2, n2 = len(rhs), n + 1
    col_ptr = np.zeros(n2 + 1, dtype=np.int32)
    ri, va = [], []
    for j, c in enumerate(cols):
        for r, v in sorted(c):
            ri.append(r)
            va.append(v)
        col_ptr[j + 1] = len(ri)
    obj = np.concatenate([base.obj, [2.5]])
    return _lp(n2, m2, col_ptr, np.array(ri, dtype=np.int32), np.array(va), obj, np.array(rhs),
               np.array(sense, dtype=np.int8), f"presolve_example_{m}x{n}_s{seed}", lb=lb, ub=ub)


class TransportFamily:
    """A fixed ns x nt transportation network whose data vary per instance: supplies x(1 + 0.2 N),
    demands x(1 + 0.2 N) rebalanced to the total supply, costs x(1 + 0.1 N) around base values
    drawn like `transport` (costs U[1,100], supplies and demand weights U{10..100}). Instance
    parameters = the concatenated multiplicative factors (ns + nt + ns*nt). Small enough (m = ns + nt
    <= 128) for the batched kernel."""

    def __init__(self, ns: int = 40, nt: int = 40, seed: int = 8):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.ns, self.nt = ns, nt
        self.base_cost = rng.uniform(1.0, 100.0, size=(ns, nt))
        self.base_supply = rng.integers(10, 101, size=ns).astype(np.float64)
        self.base_weight = rng.integers(10, 101, size=nt).astype(np.float64)

    @property
    def param_dim(self) -> int:
        return self.ns + self.nt + self.ns * self.nt

    def sample_params(self, seed: int) -> np.ndarray:
        rng = np.random.Generator(np.random.PCG64(seed))
        return np.concatenate([1.0 + 0.2 * rng.standard_normal(self.ns + self.nt),
                               1.0 + 0.1 * rng.standard_normal(self.ns * self.nt)])

    def instance(self, params: np.ndarray, name: str = "") -> Model:
        ns, nt = self.ns, self.nt
        f = np.maximum(params, 0.05)
        supply = self.base_supply * f[:ns]
        weight = self.base_weight * f[ns:ns + nt]
        demand = weight * supply.sum() / weight.sum()
        cost = self.base_cost * f[ns + nt:].reshape(ns, nt)
        return transport_structure(ns, nt, cost, supply, demand, name or f"transport_family_{ns}x{nt}")

    def instance_from_seed(self, seed: int) -> tuple[Model, np.ndarray]:
        p = self.sample_params(seed)
        return self.instance(p, f"transport_family_s{seed}"), p


class MulticommodityFamily:
    """A fixed network (nodes, arcs, capacities U[5,50], unit costs U[1,20]) with K commodities,
    each shipping from one source node to `sinks` sink nodes. Instance parameters are the
    multiplicative perturbations of sink demands (1 + 0.2 N(0,1)) and of per-(arc, commodity)
    costs (1 + 0.1 N(0,1)).

    Variables: x[a, k] (arc-major, K per arc) then nothing else; rows: `arcs` coupling rows
    sum_k x[a, k] <= cap_a, then nodes*K conservation rows out - in = supply (commodity-major)."""

    def __init__(self, nodes: int = 200, arcs: int = 1000, commodities: int = 4, sinks: int = 10,
                 seed: int = 4):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.nodes, self.arcs, self.K, self.sinks = nodes, arcs, commodities, sinks
        # a directed ring keeps every node reachable; the rest are distinct random pairs
        pairs = {(v, (v + 1) % nodes) for v in range(nodes)}
        while len(pairs) < arcs:
            u, v = rng.integers(0, nodes, size=2)
            if u != v:
                pairs.add((int(u), int(v)))
        pairs = sorted(pairs)
        rng.shuffle(pairs)
        self.tail = np.array([p[0] for p in pairs], dtype=np.int64)
        self.head = np.array([p[1] for p in pairs], dtype=np.int64)
        self.cap = rng.uniform(5.0, 50.0, size=arcs)
        self.cost = rng.uniform(1.0, 20.0, size=arcs)
        self.source = rng.choice(nodes, size=commodities, replace=False)
        self.sink_nodes = np.stack([rng.choice(np.setdiff1d(np.arange(nodes), [s]), size=sinks, replace=False)
                                    for s in self.source])
        self.base_demand = rng.uniform(2.0, 8.0, size=(commodities, sinks))
        n = arcs * commodities
        m = arcs + nodes * commodities
        a = np.repeat(np.arange(arcs), commodities)
        k = np.tile(np.arange(commodities), arcs)
        cols = np.arange(n)
        rows = np.concatenate([a, arcs + k * nodes + self.tail[a], arcs + k * nodes + self.head[a]])
        vals = np.concatenate([np.ones(n), np.ones(n), -np.ones(n)])
        self.col_ptr, self.row_idx, self.values = _csc_from_triplets(n, np.concatenate([cols, cols, cols]),
                                                                     rows, vals)
        self.n, self.m = n, m
        self.sense = np.concatenate([np.full(arcs, LE), np.full(nodes * commodities, EQ)]).astype(np.int8)

    @property
    def param_dim(self) -> int:
        return self.K * self.sinks + self.arcs * self.K

    def sample_params(self, seed: int) -> np.ndarray:
        rng = np.random.Generator(np.random.PCG64(seed))
        dem = 1.0 + 0.2 * rng.standard_normal(self.K * self.sinks)
        cst = 1.0 + 0.1 * rng.standard_normal(self.arcs * self.K)
        return np.concatenate([dem, cst])

    def instance(self, params: np.ndarray, name: str = "") -> Model:
        ks = self.K * self.sinks
        dem = self.base_demand * np.maximum(params[:ks].reshape(self.K, self.sinks), 0.05)
        cost = (np.repeat(self.cost, self.K) * np.maximum(params[ks:], 0.05))
        rhs = np.zeros(self.m)
        rhs[: self.arcs] = self.cap
        for k in range(self.K):
            base = self.arcs + k * self.nodes
            rhs[base + self.sink_nodes[k]] -= dem[k]
            rhs[base + self.source[k]] += dem[k].sum()
        return _lp(self.n, self.m, self.col_ptr, self.row_idx, self.values, cost, rhs, self.sense,
                   name or "multicommodity")

    def instance_from_seed(self, seed: int) -> tuple[Model, np.ndarray]:
        p = self.sample_params(seed)
        return self.instance(p, f"multicommodity_s{seed}"), p


# ---------------------------------------------------------------------------------------------
# The reference's own deterministic regression models (tests/unit/test_correctness_regressions.cpp)
# ---------------------------------------------------------------------------------------------

def reference_transport(m: int) -> Model:
    """build_transport(m) (test_correctness_regressions.cpp:74-111): c_ij = 1 + 0.04((7i+3j)%5),
    every supply and demand 10."""
    i = np.repeat(np.arange(m), m)
    j = np.tile(np.arange(m), m)
    cost = 1.0 + 0.04 * ((i * 7 + j * 3) % 5)
    return transport_structure(m, m, cost, np.full(m, 10.0), np.full(m, 10.0), f"reference_transport_{m}")


def reference_staircase(products: int, periods: int) -> Model:
    """build_staircase (test_correctness_regressions.cpp:157-180): make/stock per product and
    period, balance equalities and one capacity row per period."""
    names = []
    var = {}
    obj = []
    for t in range(periods):
        for p in range(products):
            for kind in ("make", "stock"):
                var[(kind, p, t)] = len(names)
                names.append((kind, p, t))
                obj.append(1.0 + 0.1 * ((p * 3 + t * 7) % 11) if kind == "make" else 0.05 + 0.01 * (p % 4))
    rows, cols, vals, rhs, sense = [], [], [], [], []
    r = 0
    for t in range(periods):
        cap_terms = []
        for p in range(products):
            terms = [(var[("make", p, t)], 1.0), (var[("stock", p, t)], -1.0)]
            if t > 0:
                terms.append((var[("stock", p, t - 1)], 1.0))
            for c, v in terms:
                rows.append(r); cols.append(c); vals.append(v)
            rhs.append(5.0 + float((p * 5 + t * 3) % 9)); sense.append(EQ); r += 1
            cap_terms.append((var[("make", p, t)], 1.0 + 0.1 * (p % 3)))
        for c, v in cap_terms:
            rows.append(r); cols.append(c); vals.append(v)
        rhs.append(12.0 * products); sense.append(LE); r += 1
    n = len(names)
    col_ptr, row_idx, values = _csc_from_triplets(n, np.array(cols), np.array(rows), np.array(vals))
    return _lp(n, r, col_ptr, row_idx, values, np.array(obj), np.array(rhs), np.array(sense, dtype=np.int8),
               f"reference_staircase_{products}x{periods}")


def reference_portfolio(assets: int, sectors: int) -> Model:
    """build_portfolio (test_correctness_regressions.cpp:263-290): diagonally dominant covariance
    with symmetric couplings, a budget equality and sector caps."""
    from collections import defaultdict
    q = defaultdict(float)
    obj = np.zeros(assets)
    for j in range(assets):
        obj[j] = -0.01 - 0.19 * ((j * 37) % 101) / 100.0
        q[(j, j)] += 0.5 + 1.5 * ((j * 53) % 97) / 96.0
        for t in range(1, 4):
            k = (j * 7 + t * 13) % assets
            if k == j:
                continue
            v = 0.05 * (((j + k * t) % 21) - 10) / 10.0
            q[(j, k)] += v
            q[(k, j)] += v
    rows, cols, vals = [], [], []
    for j in range(assets):
        rows.append(0); cols.append(j); vals.append(1.0)
    for s in range(sectors):
        for j in range(s, assets, sectors):
            rows.append(1 + s); cols.append(j); vals.append(1.0)
    col_ptr, row_idx, values = _csc_from_triplets(assets, np.array(cols), np.array(rows), np.array(vals))
    rhs = np.array([1.0] + [0.4] * sectors)
    sense = np.array([EQ] + [LE] * sectors, dtype=np.int8)
    mdl = _lp(assets, 1 + sectors, col_ptr, row_idx, values, obj, rhs, sense,
              f"reference_portfolio_{assets}x{sectors}")
    # stored terms (row name -> col name -> q), one entry per stored (row, col) key
    keys = sorted(q.keys(), key=lambda rc: (rc[1], rc[0]))
    qc = np.array([c for _, c in keys]); qr = np.array([r for r, _ in keys]); qv = np.array([q[k] for k in keys])
    mdl.q_col_ptr, mdl.q_row_idx, mdl.q_values = _csc_from_triplets(assets, qc, qr, qv)
    return mdl


def coupled_chain_qp(n: int, seed: int, block: int = 8) -> Model:
    """min 1/2 sum_i w_i (x_{i+1} - x_i)^2 + 1/2 sum_i d_i x_i^2 - t'x, 0 <= x <= 2, with
    w ~ 1 + U(0,1), d ~ 0.01 + 0.1 U(0,1), t ~ N(0,1); a covering row sum_j a_j x_j >= r_k over each
    block of `block` consecutive columns (a ~ 0.5 + U(0,1), r ~ 0.2 block U(0,1)) and the budget
    row sum_j x_j = n / 4. Strictly convex, so the primal optimum is unique."""
    rng = np.random.default_rng(seed)
    w = 1.0 + rng.random(n - 1)
    d = 0.01 + 0.1 * rng.random(n)
    t = rng.standard_normal(n)
    a = 0.5 + rng.random(n)
    nb = (n + block - 1) // block
    r = 0.2 * block * rng.random(nb)
    j = np.arange(n)
    rows = np.concatenate([j // block, np.full(n, nb)])
    cols = np.concatenate([j, j])
    vals = np.concatenate([a, np.ones(n)])
    col_ptr, row_idx, values = _csc_from_triplets(n, cols, rows, vals)
    rhs = np.concatenate([r, [n / 4.0]])
    sense = np.array([GE] * nb + [EQ], dtype=np.int8)
    mdl = _lp(n, nb + 1, col_ptr, row_idx, values, -t, rhs, sense, f"coupled_chain_qp_{n}",
              lb=np.zeros(n), ub=np.full(n, 2.0))
    diag = d.copy()
    diag[:-1] += w
    diag[1:] += w
    # stored terms: (j, j), and (j, j+1), (j+1, j) with -w_j each (the pair adds up to -w_j x_j x_{j+1})
    qc = np.concatenate([j, j[:-1], j[1:]])
    qr = np.concatenate([j, j[1:], j[:-1]])
    qv = np.concatenate([diag, -w, -w])
    mdl.q_col_ptr, mdl.q_row_idx, mdl.q_values = _csc_from_triplets(n, qc, qr, qv)
    return mdl


def free_intercept_qp(points: int, features: int, seed: int) -> Model:
    """Ridge regression with a free intercept: min 1/2 ||r||^2 + lam/2 ||beta||^2 subject to
    r_i + X_i beta + b0 = y_i, -1 <= beta_k <= 1, r and b0 free; X ~ N(0,1), y = X beta0 + 3 + noise,
    lam = 0.1. The intercept b0 is free and carries no curvature: its column of the Hessian is zero."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((points, features))
    beta0 = rng.uniform(-1.5, 1.5, features)
    y = X @ beta0 + 3.0 + 0.1 * rng.standard_normal(points)
    n = points + features + 1  # r, beta, b0
    rows, cols, vals = [], [], []
    i = np.arange(points)
    rows.append(i); cols.append(i); vals.append(np.ones(points))
    for k in range(features):
        rows.append(i); cols.append(np.full(points, points + k)); vals.append(X[:, k])
    rows.append(i); cols.append(np.full(points, n - 1)); vals.append(np.ones(points))
    col_ptr, row_idx, values = _csc_from_triplets(n, np.concatenate(cols), np.concatenate(rows),
                                                  np.concatenate(vals))
    lb = np.concatenate([np.full(points, -INF), np.full(features, -1.0), [-INF]])
    ub = np.concatenate([np.full(points, INF), np.full(features, 1.0), [INF]])
    mdl = _lp(n, points, col_ptr, row_idx, values, np.zeros(n), y, np.full(points, EQ, dtype=np.int8),
              f"free_intercept_qp_{points}x{features}", lb=lb, ub=ub)
    jq = np.arange(points + features)
    qv = np.concatenate([np.ones(points), np.full(features, 0.1)])
    mdl.q_col_ptr, mdl.q_row_idx, mdl.q_values = _csc_from_triplets(n, jq, jq, qv)
    return mdl


def small_qp_offdiagonal() -> Model:
    """QpAccuracy.OffDiagonalHessianTermsCountOnce (test_correctness_regressions.cpp:221-245):
    min 1/2(2x^2 + xy + 2y^2) - x - y, x + y <= 5, 0 <= x, y <= 10; optimum x = y = 0.4, -0.4."""
    col_ptr = np.array([0, 1, 2], dtype=np.int32)
    mdl = _lp(2, 1, col_ptr, np.array([0, 0], dtype=np.int32), np.array([1.0, 1.0]), np.array([-1.0, -1.0]),
              np.array([5.0]), np.array([LE], dtype=np.int8), "qp_offdiagonal", lb=np.zeros(2),
              ub=np.full(2, 10.0))
    # stored terms: (x,x)=2, (x,y)=1 [row x, col y], (y,y)=2
    mdl.q_col_ptr = np.array([0, 1, 3], dtype=np.int32)
    mdl.q_row_idx = np.array([0, 0, 1], dtype=np.int32)
    mdl.q_values = np.array([2.0, 1.0, 2.0])
    return mdl


def bounded_lp_example() -> Model:
    """A small LP exercising every branch of the standard-form conversion: maximize, Le/Ge/Eq rows,
    nonzero lower bounds, finite upper bounds (extra rows), and an objective constant."""
    # max 3x0 + 2x1 - x2 + 4 ; x0 + x1 + x2 <= 10 ; x0 - x1 >= -2 ; x1 + 2 x2 == 6
    # 1 <= x0 <= 6, 0 <= x1, 0.5 <= x2 <= 4
    cols = np.array([0, 0, 1, 1, 1, 2, 2])
    rows = np.array([0, 1, 0, 1, 2, 0, 2])
    vals = np.array([1.0, 1.0, 1.0, -1.0, 1.0, 1.0, 2.0])
    col_ptr, row_idx, values = _csc_from_triplets(3, cols, rows, vals)
    mdl = _lp(3, 3, col_ptr, row_idx, values, np.array([3.0, 2.0, -1.0]), np.array([10.0, -2.0, 6.0]),
              np.array([LE, GE, EQ], dtype=np.int8), "bounded_lp", lb=np.array([1.0, 0.0, 0.5]),
              ub=np.array([6.0, INF, 4.0]), constant=4.0)
    mdl.maximize = True
    return mdl
