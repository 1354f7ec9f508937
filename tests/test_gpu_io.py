"""Checkpoint and dump files written while the lattice keeps stepping
(lb3dc_checkpoint_async, lb3dc_dump_async): byte-equal to the synchronous
download + XDR writers at the step the write was started."""
import numpy as np
import pytest

from lb3d_b200.config import Params
from lb3d_b200.ic import uniform_mixture

pytestmark = pytest.mark.gpu


def _params(dims, nc, precision, **kw):
    base = dict(nx=dims[0], ny=dims[1], nz=dims[2], ncomp=nc, tau_d=1.0, g_br=0.08, g_bs=-0.006,
                g_ss=-0.0045, beta=10.0, d_0=1.0, bdist=2, restore=1, precision=precision)
    base.update(kw)
    return Params(**base).finalize()


@pytest.mark.parametrize("nc,precision", [(3, 0), (3, 1), (2, 0)])
def test_async_checkpoint_and_dumps_equal_synchronous_files(nc, precision, tmp_path):
    from lb3d_b200.lib import Lattice, write_checkpoint, write_field
    dims = (12, 10, 9)
    st = uniform_mixture(*dims, nc, seed=29)
    rock = None
    if nc == 2:
        rock = np.zeros(dims[::-1])
        rock[2, 3, 4:7] = 1.0
        st["rock"] = rock
    lat = Lattice(_params(dims, nc, precision), precision=precision)
    lat.upload_state(st)
    lat.time_loop(5)
    ref = lat.download()
    lat.checkpoint_async(tmp_path / "a.xdr")
    lat.time_loop(7)  # steps while the file is written
    lat.io_wait()
    write_checkpoint(str(tmp_path / "s.xdr"), ref["n"], db=ref["db"] if nc == 3 else None,
                     rock=rock, da=ref["da"] if nc == 3 else None)
    assert (tmp_path / "a.xdr").read_bytes() == (tmp_path / "s.xdr").read_bytes()
    for field, k in (("od", 1), ("vel", 1), ("arr", 3)):
        want = lat.dump(field)
        lat.dump_async(field, tmp_path / f"a_{field}.xdr", dump_double=(field == "vel"))
        lat.time_loop(2)
        lat.io_wait()
        write_field(str(tmp_path / f"s_{field}.xdr"), want, k, dump_double=(field == "vel"))
        assert (tmp_path / f"a_{field}.xdr").read_bytes() == (tmp_path / f"s_{field}.xdr").read_bytes()
    lat.close()


def test_async_write_error_is_reported(tmp_path):
    from lb3d_b200.lib import Lattice, Lb3dError
    dims = (8, 8, 8)
    lat = Lattice(_params(dims, 2, 0), precision=0)
    lat.upload_state(uniform_mixture(*dims, 2, seed=1))
    lat.checkpoint_async(tmp_path / "no_such_dir" / "c.xdr")
    lat.time_loop(1)
    with pytest.raises(Lb3dError):
        lat.io_wait()
    lat.io_wait()  # the error is reported once
    lat.close()
