"""Multi-GPU plumbing: one process per GPU, replicas only.

The hot path exchanges no data between independent lattices, so N GPUs run
N independent lattices (or N disjoint shares of a request stream) with no
collective on the data path.  torch.distributed is used only to agree on
timing: a barrier before and after the timed region and the maximum of the
per-rank device times.  Ranks read RANK / LOCAL_RANK / WORLD_SIZE /
MASTER_ADDR / MASTER_PORT from the environment (torchrun).
"""
from __future__ import annotations

import datetime
import os
from typing import List, Sequence, TypeVar

T = TypeVar("T")


def world() -> tuple:
    """(rank, local_rank, world_size) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """Initialises the process group when WORLD_SIZE > 1; returns it or None."""
    import torch.distributed as dist
    rank, local, size = world()
    if size <= 1:
        return None
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def partition(items: Sequence[T], rank: int, size: int) -> List[T]:
    """This rank's share of a request stream: round-robin by position, so
    every rank sees arrivals spread over the whole stream and the shares
    differ in length by at most one."""
    if size < 1 or not (0 <= rank < size):
        raise ValueError("bad rank/size")
    return [x for i, x in enumerate(items) if i % size == rank]


def max_over_ranks(values: Sequence[float], device: str = "cpu") -> List[float]:
    """Element-wise maximum over ranks (the job's time is its slowest rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def sum_over_ranks(values: Sequence[float], device: str = "cpu") -> List[float]:
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu()]


def replica_seed(base_seed: int, rank: int) -> int:
    """Seed of a rank's replica lattice: distinct and reproducible."""
    return base_seed + 7919 * rank
