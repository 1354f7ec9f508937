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


def _slab_worker(rank, size, port, nc, dims, steps, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(size),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import dataclasses
    import numpy as np
    import torch
    import torch.distributed as dist
    from tests._oracle import Oracle
    D.init("gloo", timeout_s=120)
    p, st = _slab_case(nc, dims)
    y0, ny = D.y_slab(p.ny, rank, size)
    sl = slice(y0, y0 + ny)
    mine = dict(n=st["n"][:, :, :, sl], db=None if st["db"] is None else st["db"][:, :, sl],
                rock=st["rock"][:, sl], shear_sum=0.0)

    def exchange(o):
        lo = torch.from_numpy(o.yplane(1))
        hi = torch.from_numpy(o.yplane(ny))
        lower, upper = D.exchange_y_faces(lo, hi, rank, size)
        o.set_yplane(0, lower.numpy())
        o.set_yplane(ny + 1, upper.numpy())

    o = Oracle(dataclasses.replace(p, ny=ny), mine, threads=1, slab=(y0, exchange))
    o.run(steps)
    g = o.get()
    out[rank] = (y0, ny, g["n"], g["db"])
    dist.barrier()
    dist.destroy_process_group()


def _slab_case(nc, dims):
    import numpy as np
    from lb3d_b200.config import Params
    from lb3d_b200.ic import uniform_mixture
    kw = dict(tau_d=1.0, g_br=0.08, beta=10.0, d_0=1.0, bdist=2, restore=1,
              g_accn=1e-4, g_accn_y=3e-5, g_accn_min_y=3, g_accn_max_y=6)
    if nc == 3:
        kw.update(g_bs=-0.006, g_ss=-0.0045)
    else:
        kw.update(g_wr=-0.1, g_wb=0.05, rock_colour_r=1.0, rock_colour_b=0.5)
    p = Params(nx=dims[0], ny=dims[1], nz=dims[2], ncomp=nc, **kw).finalize()
    st = uniform_mixture(*dims, nc, seed=41)
    if nc == 2:
        rng = np.random.default_rng(2)
        st["rock"] = (rng.random(st["n"].shape[2:]) < 0.15).astype(np.float64)
    return p, st


@pytest.mark.parametrize("nc,dims", [(3, (6, 9, 5)), (2, (7, 8, 6))])
def test_y_slabs_over_two_gloo_ranks_equal_one_lattice(nc, dims):
    """One lattice split into two y-slabs, each stepped by its own oracle on
    its own rank; the y faces travel between the ranks (point to point,
    periodic over the ranks) at every halo exchange of the step.  After the
    steps the slabs put together equal the single-lattice oracle bit for
    bit: every site sees the same neighbours in the same order, the body
    force region is evaluated in global coordinates (a y sub-range that
    crosses the slab boundary), and walls cross it too (binary case)."""
    import numpy as np
    from tests._oracle import Oracle
    size, steps = 2, 6
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_slab_worker, args=(size, port, nc, dims, steps, out), nprocs=size, join=True)
        parts = dict(out)
    p, st = _slab_case(nc, dims)
    o = Oracle(p, st, threads=1)
    o.run(steps)
    ref = o.get()
    for rank in range(size):
        y0, ny, n, db = parts[rank]
        np.testing.assert_array_equal(n, ref["n"][:, :, :, y0:y0 + ny])
        if nc == 3:
            np.testing.assert_array_equal(db, ref["db"][:, :, y0:y0 + ny])


def test_y_slab_split():
    assert [D.y_slab(10, r, 3) for r in range(3)] == [(0, 3), (3, 3), (6, 4)]
    assert sum(D.y_slab(128, r, 8)[1] for r in range(8)) == 128
    with pytest.raises(ValueError):
        D.y_slab(2, 0, 3)
