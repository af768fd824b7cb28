"""Multi-GPU plumbing for independent replicas (one process per GPU).

The solver's path has no exchange step: a single program runs on one GPU and
a batch of programs splits into independent shards.  N > 1 therefore means N
processes that each solve their own work, with only host-side bookkeeping
collectives: a barrier around timed regions, the maximum of the ranks' times
and the sum of the work they did.  The process group is gloo (CPU tensors):
nothing on the solve path depends on it.
"""
from __future__ import annotations

import datetime
import os
from typing import Sequence, TypeVar

T = TypeVar("T")


def env():
    """(rank, world, local_rank) from the torchrun environment (1 process if unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(world: int, timeout_s: float = 600.0) -> None:
    if world > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))


def finalize(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(value: float, world: int, op: str) -> float:
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t[0])


def max_over_ranks(value: float, world: int) -> float:
    """The job's time: the slowest rank's."""
    return _reduce(value, world, "max")


def sum_over_ranks(value: float, world: int) -> float:
    """The job's work: every rank's units added up."""
    return _reduce(value, world, "sum")


def shard(items: Sequence[T], rank: int, world: int) -> list:
    """Round-robin share of a batch for one rank (every item on exactly one rank)."""
    return [items[i] for i in range(rank, len(items), world)]
