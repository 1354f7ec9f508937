"""Replica plumbing across ranks, run as two gloo processes on the CPU:
request partitioning covers the stream exactly once, and timing agrees on
the slowest rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from lb3d_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, size, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(size),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    from lb3d_b200.ensemble import sweep_requests
    D.init("gloo", timeout_s=60)
    reqs = sweep_requests(101, seed=4)
    mine = D.partition(reqs, rank, size)
    ids = torch.zeros(101, dtype=torch.int64)
    for r in mine:
        ids[r.rid] += 1
    dist.all_reduce(ids)
    t = D.max_over_ranks([1.0 + rank, 5.0 - rank])
    n = D.sum_over_ranks([len(mine)])[0]
    out[rank] = (ids.tolist(), t, n, D.replica_seed(1, rank))
    dist.barrier()
    dist.destroy_process_group()


def test_partition_and_max_over_two_gloo_ranks():
    size = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(size, port, out), nprocs=size, join=True)
        res = dict(out)
    for rank in range(size):
        ids, t, n, seed = res[rank]
        assert ids == [1] * 101  # every request on exactly one rank
        assert t == [2.0, 5.0]
        assert n == 101
    assert res[0][3] != res[1][3]


def test_partition_single_process():
    assert D.partition(list(range(7)), 1, 3) == [1, 4]
    with pytest.raises(ValueError):
        D.partition([1], 3, 3)
