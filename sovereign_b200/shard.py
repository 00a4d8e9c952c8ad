"""Multi-GPU plumbing for batches of independent LPs.

Independent LPs shard with no data-path collective. Two ways:

* ``solve_batch_sharded``: one caller list held by every rank (one process per GPU, torchrun) is
  split by size bucket (the batched kernel's 32-row buckets of IPM rows, then the LPs it hands to the
  single-problem engine), each bucket's LPs dealt to the ranks by estimated cost (largest first, to
  the least-loaded rank), so every rank gets a share of every bucket. The split is a pure function
  of the list, so the ranks agree on it without communicating. Each rank solves its share with one
  batched call on its own GPU; the results are gathered to one rank on the host and put back in the
  caller's order. This is the multi-GPU counterpart of N independent InteriorPointSolver::solve
  calls (solver/milp/src/branch_and_bound.cpp:497).
* the benchmark's weak scaling: every rank solves its own LPs (instance seeds offset by rank).

The only communication is host-side: the result gather, a barrier around a timed region and the
maximum device time over ranks. torch.distributed carries it (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import os

import numpy as np

from . import abi


def world() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the torchrun environment (1 process by default)."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def shard_seed(base: int, rank: int) -> int:
    """Seed of rank's shard: disjoint instance streams per rank."""
    return base + rank


def shard_range(count: int, rank: int, world_size: int) -> range:
    """Contiguous, balanced split of count items (used when one list is spread over ranks)."""
    per, extra = divmod(count, world_size)
    start = rank * per + min(rank, extra)
    return range(start, start + per + (1 if rank < extra else 0))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar (device time) over all ranks; identity without a process group."""
    if dist is None or not dist.is_initialized():
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None or not dist.is_initialized():
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


BATCH_MAX_ROWS = 128   # IPM rows the batched kernel takes (larger LPs go to the single engine)
BUCKET_ROWS = 32       # the batched kernel's bucket granularity


def ipm_shape(model) -> tuple[int, int]:
    """(IPM columns, IPM rows) of an LP after the standard form (interior_point.cpp:224-409): every
    finite upper bound adds a row and a slack column, every inequality row a slack column."""
    ub = np.asarray(model.ub)
    n_ub = int(np.sum(np.isfinite(ub) & (ub < 1e29)))
    n_slack = int(np.sum(np.asarray(model.sense) != abi.EQ)) + n_ub
    return model.n + n_slack, model.m + n_ub


def bucket_of(m_ipm: int) -> int:
    """Size bucket of an LP: 32, 64, 96 or 128 IPM rows for the batched kernel, 0 for the LPs the
    single-problem engine solves (empty, or more rows than the batched kernel takes)."""
    if m_ipm <= 0 or m_ipm > BATCH_MAX_ROWS:
        return 0
    return max(BUCKET_ROWS, -(-m_ipm // BUCKET_ROWS) * BUCKET_ROWS)


def lp_cost(model) -> float:
    """Relative cost of one LP: the dense factorization (m^3 / 3) plus the passes over A."""
    n_ipm, m_ipm = ipm_shape(model)
    return m_ipm ** 3 / 3.0 + 16.0 * (model.nnz + n_ipm) + 1.0


def partition(models, world_size: int) -> list[list[int]]:
    """Indices of `models` for each rank, ascending. Within every size bucket the LPs go largest
    first to the rank with the least work in that bucket (ties: least work overall, then lowest
    rank). Deterministic: every rank computes the same split."""
    buckets: dict[int, list[tuple[float, int]]] = {}
    for i, mdl in enumerate(models):
        buckets.setdefault(bucket_of(ipm_shape(mdl)[1]), []).append((lp_cost(mdl), i))
    parts: list[list[int]] = [[] for _ in range(world_size)]
    total = [0.0] * world_size
    for key in sorted(buckets):
        load = [0.0] * world_size
        for cost, i in sorted(buckets[key], key=lambda t: (-t[0], t[1])):
            r = min(range(world_size), key=lambda q: (load[q], total[q], q))
            parts[r].append(i)
            load[r] += cost
            total[r] += cost
    for p in parts:
        p.sort()
    return parts


def solve_batch_sharded(models, options=None, dist=None, root: int = 0, solver=None, **kwargs):
    """Solve one list of independent LPs spread over the ranks of `dist` (one GPU per rank), the
    results gathered to `root` in the caller's order; other ranks get None. Every rank passes the
    same list. Without a process group this is one batched call. `solver(models, options, **kwargs)`
    defaults to sovereign_b200.ipm.solve_batch (sov_lp_solve_batch on this rank's current device)."""
    if solver is None:
        from .ipm import solve_batch as solver
    if dist is None or not dist.is_initialized():
        return solver(list(models), options, **kwargs)
    rank, world_size = dist.get_rank(), dist.get_world_size()
    mine = partition(models, world_size)[rank]
    res = solver([models[i] for i in mine], options, **kwargs) if mine else []
    payload = list(zip(mine, res))
    gathered = [None] * world_size if rank == root else None
    dist.gather_object(payload, gathered, dst=root)
    if rank != root:
        return None
    out = [None] * len(models)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
