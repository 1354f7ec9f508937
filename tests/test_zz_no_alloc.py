"""The FP64 step without device allocation (lb3dc_time_loop_fp64_noalloc).

Callers that may not call cudaMalloc (every device byte owned by the
caller's own pool or arrays) hand the step their own device buffers; its scratch lives in a
fixed-size device array inside the library.  Its results must be those of
the allocating entry point: the FP64 path is exact, so the comparison is
exact, over two calls in a row (the scratch array keeps the previous call's
bytes).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from lb3d_b200.config import Params, to_cparams
from lb3d_b200.ic import uniform_mixture

pytestmark = pytest.mark.gpu


def _noalloc(p, f, db, rock, nsteps, stream):
    from lb3d_b200.lib import lib
    L = lib()
    fn = L.lb3dc_time_loop_fp64_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(type(to_cparams(p))), ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    cp = to_cparams(p)
    return fn(ctypes.byref(cp), f, db, rock, nsteps, stream)


def _last_error():
    from lb3d_b200.lib import lib
    buf = ctypes.create_string_buffer(512)
    lib().lb3dc_last_error(None, buf, 512)
    return buf.value.decode()


@pytest.mark.parametrize("nc,dims,with_rock", [(3, (20, 18, 16), False), (2, (24, 20, 18), True)])
def test_noalloc_matches_allocating_entry_point(nc, dims, with_rock):
    import torch
    from lb3d_b200.lib import Lattice

    p = Params(nx=dims[0], ny=dims[1], nz=dims[2], ncomp=nc, tau_d=1.0, g_br=0.08, g_bs=-0.006,
               g_ss=-0.0045, beta=10.0, d_0=1.0, bdist=2, restore=1, g_wr=-0.05, rock_colour_r=1.0,
               g_accn_x=1e-4).finalize()
    st = uniform_mixture(*dims, nc, seed=21)
    rock = None
    if with_rock:
        rng = np.random.default_rng(2)
        rock = (rng.random(st["n"].shape[2:]) < 0.15).astype(np.float64)
        st["rock"] = rock
        st["n"] = np.where(rock[None, None] != 0, 0.0, st["n"])  # lbe_init_rock_colour

    # the allocating entry point
    lat = Lattice(p, precision=0)
    lat.upload_state(st)
    lat.time_loop(7)
    ref1 = lat.download()
    lat.time_loop(5)
    ref2 = lat.download()
    lat.close()

    # the same steps through the no-alloc entry point on caller-owned buffers
    dev = torch.device("cuda")
    f = torch.from_numpy(np.ascontiguousarray(st["n"])).to(dev)
    db = torch.from_numpy(np.ascontiguousarray(st["db"])).to(dev) if nc == 3 else None
    rk = torch.from_numpy(rock.astype(np.uint8)).to(dev) if with_rock else None
    s = torch.cuda.Stream()
    args = (f.data_ptr(), db.data_ptr() if db is not None else None,
            rk.data_ptr() if rk is not None else None)
    torch.cuda.synchronize()
    assert _noalloc(p, *args, 7, s.cuda_stream) == 0, _last_error()
    s.synchronize()
    np.testing.assert_array_equal(f.cpu().numpy(), ref1["n"])
    if nc == 3:
        np.testing.assert_array_equal(db.cpu().numpy(), ref1["db"])
    assert _noalloc(p, *args, 5, s.cuda_stream) == 0, _last_error()
    s.synchronize()
    np.testing.assert_array_equal(f.cpu().numpy(), ref2["n"])
    if nc == 3:
        np.testing.assert_array_equal(db.cpu().numpy(), ref2["db"])


def test_noalloc_rejects_lattices_beyond_its_scratch():
    import torch
    p = Params(nx=40, ny=40, nz=40, ncomp=3, tau_d=1.0, bdist=2).finalize()
    f = torch.zeros(1, device="cuda", dtype=torch.float64)
    rc = _noalloc(p, f.data_ptr(), f.data_ptr(), None, 1, None)
    assert rc == -22
    assert "scratch bytes" in _last_error()
