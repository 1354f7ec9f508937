"""Multi-GPU plumbing: one process per GPU.

Replicas: independent lattices exchange no data, so N GPUs run N
independent lattices (or N disjoint shares of a request stream) with no
collective on the data path; torch.distributed only agrees on timing (a
barrier around the timed region and the maximum of the per-rank device
times).

Slabs: one lattice split along y over the ranks, as the reference splits its
lattice over MPI ranks (code/lb3d_mpi.F90:492-596).  Each rank owns a
contiguous range of y planes (y_slab) and, at every halo exchange, sends its
first plane to the rank below and its last plane to the rank above and
receives their faces into its y-halo planes (exchange_y_faces), periodic in
y across the ranks.  The faces travel point to point (NCCL over NVLink on
GPUs, gloo on the CPU).

Ranks read RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT from
the environment (torchrun).
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


def y_slab(ny: int, rank: int, size: int) -> tuple:
    """(y0, planes) of this rank's slab: ny planes split into contiguous
    ranges that differ in length by at most one (each at least one plane)."""
    if size < 1 or not (0 <= rank < size) or ny < size:
        raise ValueError("bad rank/size for the slab split")
    y0 = ny * rank // size
    return y0, ny * (rank + 1) // size - y0


# message tags of the two faces: a rank's last plane becomes the lower halo
# of the rank above, its first plane the upper halo of the rank below
_TAG_TO_ABOVE, _TAG_TO_BELOW = 17, 18


def exchange_y_faces(lo, hi, rank: int, size: int, group=None):
    """Sends this slab's first (lo) and last (hi) y planes to the ranks below
    and above and returns (lower_halo, upper_halo): the plane below y = 0
    (the last plane of the rank below) and the plane above the last one (the
    first plane of the rank above), periodic over the ranks.  lo, hi: torch
    tensors of one plane each (any device the backend supports)."""
    import torch
    import torch.distributed as dist
    if size == 1:
        return hi.clone(), lo.clone()
    below, above = (rank - 1) % size, (rank + 1) % size
    lower, upper = torch.empty_like(hi), torch.empty_like(lo)
    ops = [dist.P2POp(dist.isend, hi.contiguous(), above, group, _TAG_TO_ABOVE),
           dist.P2POp(dist.isend, lo.contiguous(), below, group, _TAG_TO_BELOW),
           dist.P2POp(dist.irecv, lower, below, group, _TAG_TO_ABOVE),
           dist.P2POp(dist.irecv, upper, above, group, _TAG_TO_BELOW)]
    for w in dist.batch_isend_irecv(ops):
        w.wait()
    return lower, upper
