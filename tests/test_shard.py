"""The N>1 path of bench.py on CPU: two gloo ranks shard the batched workload without overlap, time
with max over ranks and count the whole job (no GPU, no collective on the data path)."""
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
