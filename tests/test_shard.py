"""The N>1 paths on CPU (no GPU, no collective on the data path): two gloo ranks shard the batched
workload without overlap, time with max over ranks and count the whole job; and one caller list is
split by size bucket over the ranks, solved per rank and gathered back in the caller's order
(solve_batch_sharded, with the oracle restatement standing in for the GPU solve)."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from sovereign_b200 import shard  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from sovereign_b200 import problems as P
    models = P.transport_batch(6, seed=shard.shard_seed(2026, rank))
    sig = [float(m.obj.sum()) for m in models]
    local_time = 1.0 + rank  # stands in for this rank's device time
    t = shard.max_over_ranks(local_time, dist)
    total = shard.sum_over_ranks(len(models), dist)
    gathered = [None] * world
    dist.all_gather_object(gathered, sig)
    out[rank] = (t, total, gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_and_timing():
    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        t, total, gathered = res[rank]
        assert t == 2.0            # max over ranks, the job's time
        assert total == 12         # whole-job count for the throughput
        a, b = gathered
        assert not set(a) & set(b)  # disjoint shards


def test_shard_range_balanced():
    parts = [shard.shard_range(10, r, 3) for r in range(3)]
    assert [len(p) for p in parts] == [4, 3, 3]
    assert sorted(i for p in parts for i in p) == list(range(10))


def _oracle_solver(models, options=None, **kw):
    import oracle
    return [oracle.solve(m, kind="restatement") for m in models]


def _mixed_list():
    from sovereign_b200 import problems as P
    return (P.transport_batch(9, seed=41) + [P.transport(70, 80, 3)] + P.transport_batch(5, seed=42) +
            [P.reference_staircase(8, 40), P.random_sparse_lp(30, 90, 3, 8)])


def _sharded_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    models = _mixed_list()
    res = shard.solve_batch_sharded(models, dist=dist, solver=_oracle_solver)
    out[rank] = None if res is None else [(r.status, r.objective_value) for r in res]
    dist.barrier()
    dist.destroy_process_group()


def test_partition_by_bucket_covers_and_balances():
    models = _mixed_list()
    for world in (1, 2, 3, 4):
        parts = shard.partition(models, world)
        assert sorted(i for p in parts for i in p) == list(range(len(models)))
        assert all(p == sorted(p) for p in parts)
        assert parts == shard.partition(models, world)  # deterministic
        buckets = {}
        for i, m in enumerate(models):
            buckets.setdefault(shard.bucket_of(shard.ipm_shape(m)[1]), []).append(i)
        for key, idx in buckets.items():  # every bucket with enough LPs is spread over every rank
            if len(idx) >= world:
                assert all(any(i in p for i in idx) for p in parts), (world, key)
    # LPs beyond the batched kernel's rows (and empty ones) form the single-engine bucket
    assert shard.bucket_of(129) == 0 and shard.bucket_of(0) == 0 and shard.bucket_of(33) == 64


def test_two_rank_split_solve_and_gather():
    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_sharded_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[1] is None
    want = [(r.status, r.objective_value) for r in _oracle_solver(_mixed_list())]
    assert res[0] == want  # every LP back, in the caller's order, solved exactly once
