"""Multi-GPU plumbing for batches of independent LPs.

The batched workload shards with no data-path collective: every rank solves its own LPs (instance
seeds offset by rank, so shards never overlap), and the only communication is timing and result
bookkeeping on the host side: a barrier around the timed region and the maximum device time over
ranks. torch.distributed carries it (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import os


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
