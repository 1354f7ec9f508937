"""The C-ABI library: it loads, exports every entry point include/lb3dc.h
declares, validates parameters before touching a device, and its host-side
pieces (XDR codec, deterministic math) work without a GPU."""
import os
import re

import numpy as np
import pytest

from lb3d_b200 import lib as L
from lb3d_b200.config import Params
from tests._fixtures import GOLDEN, STAMP, load_case, read_gz

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(lb3dc_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L.lib()
    import ctypes
    so = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(so, n)]
    assert not missing, missing
    assert len(declared_symbols()) >= 30
    assert b"sm_100a" in L.lib().lb3dc_version()


def test_create_rejects_fatal_combinations_before_device():
    p = Params(nx=8, ny=8, nz=8, ncomp=3, bdist=2, boundary_cond=-1, inv_fluid=5).finalize()
    with pytest.raises(ValueError):
        p.validate()
    import ctypes
    from lb3d_b200.config import to_cparams
    cp = to_cparams(p)
    h = ctypes.c_void_p()
    rc = L.lib().lb3dc_create(ctypes.byref(cp), ctypes.byref(h))
    assert rc == L.LB3DC_EINVAL
    buf = ctypes.create_string_buffer(256)
    L.lib().lb3dc_last_error(None, buf, 256)
    assert b"Lees Edwards" in buf.value
    assert L.lib().lb3dc_footprint(ctypes.byref(cp)) == -1


def test_footprint():
    p = Params(nx=32, ny=32, nz=32, ncomp=3, bdist=2).finalize()
    N = 32 ** 3
    fb = L.footprint(p)
    assert fb >= 2 * 3 * 19 * N * 8
    p.precision = 1
    # half the population bytes, plus the moment-field strategy's padded
    # fields (48 B per site) when every component relaxes fully
    assert L.footprint(p) < fb / 1.7


@pytest.mark.parametrize("case", ["gyroid", "wettingWall"])
def test_xdr_checkpoint_roundtrip(case, tmp_path):
    p, st = load_case(case)
    raw = read_gz(os.path.join(GOLDEN, case, f"checkpoint_{case}_{STAMP}_p000000.xdr"))
    src = tmp_path / "in.xdr"
    src.write_bytes(raw)
    got = L.read_checkpoint(str(src), p.nx, p.ny, p.nz, p.ncomp)
    np.testing.assert_array_equal(got["n"], st["n"])
    if p.ncomp == 3:
        np.testing.assert_array_equal(got["db"], st["db"])
    # writing back reproduces the reference's bytes (da is written equal to
    # the restored da, which the test checkpoints store equal to db)
    nd = 64 if p.ncomp == 3 else 39
    cp = np.frombuffer(raw, ">f8").reshape(p.nx, p.ny, p.nz, nd).transpose(2, 1, 0, 3)
    da = np.ascontiguousarray(cp[..., 57:60].transpose(3, 0, 1, 2)) if p.ncomp == 3 else None
    out = tmp_path / "out.xdr"
    L.write_checkpoint(str(out), got["n"], got["db"], got["rock"], da=da)
    assert out.read_bytes() == raw


def test_xdr_topo_rock_and_fields(tmp_path):
    raw = read_gz(os.path.join(GOLDEN, "leesEdwards", f"checktopo_leesEdwards_{STAMP}.xdr"))
    (tmp_path / "t.xdr").write_bytes(raw)
    ss = L.read_topo(str(tmp_path / "t.xdr"))
    assert abs(ss - 0.01 * 16 / 15) < 1e-7
    L.write_topo(str(tmp_path / "t2.xdr"), ss)
    assert (tmp_path / "t2.xdr").read_bytes() == raw
    wall = read_gz(os.path.join(GOLDEN, "wettingWall", "wettingWall.wall.xdr"))
    (tmp_path / "w.xdr").write_bytes(wall)
    rock = L.read_rock(str(tmp_path / "w.xdr"), 16, 16, 16)
    assert rock.sum() == 256 and rock[0].all()
    L.write_rock(str(tmp_path / "w2.xdr"), rock)
    assert (tmp_path / "w2.xdr").read_bytes() == wall
    v = np.linspace(-1, 1, 30)
    L.write_field(str(tmp_path / "f.xdr"), v, values_per_site=3)
    np.testing.assert_array_equal(np.frombuffer((tmp_path / "f.xdr").read_bytes(), ">f4"), v.astype(np.float32))


def _ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    ia = np.where(ia < 0, np.int64(-0x8000000000000000) - ia, ia)
    ib = np.where(ib < 0, np.int64(-0x8000000000000000) - ib, ib)
    return np.abs(ia - ib)


def test_detmath_host_accuracy():
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(-20, 20, 200000), rng.uniform(-1, 1, 200000),
                        rng.uniform(-700, 700, 20000), -np.abs(rng.normal(0.7, 0.3, 200000))])
    e = L.detmath_eval("exp", x)
    assert _ulps(e, np.exp(x)).max() <= 2
    xs = rng.uniform(-0.34, 0.34, 200000)
    assert _ulps(L.detmath_eval("expm1", xs), np.expm1(xs)).max() <= 2
    t = rng.uniform(0.005, 30, 200000)
    assert _ulps(L.detmath_eval("tanh", t), np.tanh(t)).max() <= 3
    assert L.detmath_eval("exp", np.array([0.0, -np.inf, np.inf, 800.0, -800.0])).tolist() == [1.0, 0.0, np.inf, np.inf, 0.0]


def test_fp32_size_limit_checked_at_creation():
    import ctypes
    from lb3d_b200.config import to_cparams
    p = Params(nx=620, ny=620, nz=620, ncomp=3, bdist=2).finalize()
    p.validate()  # FP64 is bounded by memory only
    p.precision = 1
    with pytest.raises(ValueError):
        p.validate()
    cp = to_cparams(p)
    h = ctypes.c_void_p()
    assert L.lib().lb3dc_create(ctypes.byref(cp), ctypes.byref(h)) == L.LB3DC_EINVAL
    buf = ctypes.create_string_buffer(256)
    L.lib().lb3dc_last_error(None, buf, 256)
    assert b"FP32 lattices are limited" in buf.value
    # the largest FP32 ternary lattice the offsets allow holds 117 GB
    p2 = Params(nx=608, ny=608, nz=608, ncomp=3, bdist=2, precision=1).finalize()
    p2.validate()


@pytest.mark.parametrize("kw,text", [
    (dict(ncomp=3, inv_fluid=7), b"binary builds only"),
    (dict(ncomp=2, inv_fluid=11, nz=1), b"two distinct z planes"),
    (dict(ncomp=2, inv_fluid=12, nz=1), b"two distinct z planes"),
    (dict(ncomp=2, inv_fluid=8, nz=1), b"two z planes"),
    (dict(ncomp=2, inv_fluid=12, inv_type=2), b"inv_type"),
    (dict(ncomp=2, inv_fluid=13), b"not implemented"),
])
def test_inflow_boundaries_refused_before_device(kw, text):
    """The stage-8 inflow boundaries' invalid combinations are refused by
    lb3dc_create with LB3DC_EINVAL or LB3DC_ENOTSUP before any device work,
    on both paths."""
    import ctypes
    from lb3d_b200.config import to_cparams
    base = dict(nx=8, ny=8, nz=8, bdist=2, boundary_cond=-1)
    base.update(kw)
    for precision in (0, 1):
        p = Params(**base).finalize()
        p.precision = precision
        cp = to_cparams(p)
        h = ctypes.c_void_p()
        rc = L.lib().lb3dc_create(ctypes.byref(cp), ctypes.byref(h))
        assert rc in (L.LB3DC_EINVAL, L.LB3DC_ENOTSUP)
        buf = ctypes.create_string_buffer(256)
        L.lib().lb3dc_last_error(None, buf, 256)
        assert text in buf.value, buf.value
