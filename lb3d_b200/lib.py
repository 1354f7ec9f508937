"""ctypes binding of liblb3dc.so (include/lb3dc.h) and a Lattice class whose
methods mirror the calls lb3d_time_loop makes (code/lb3d_time_loop.F90:58-92).

The CUDA library is the only implementation: there is no CPU fallback, and
loading fails loudly when the in-tree build (lb3d_b200/_lib/liblb3dc.so) is
missing.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from .config import CParams, Params, to_cparams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liblb3dc.so")

LB3DC_OK = 0
LB3DC_EINVAL = -22
LB3DC_ENOMEM = -12
LB3DC_ECUDA = -5
LB3DC_ETIMEOUT = -110
LB3DC_ENAN = -33
LB3DC_ENOTSUP = -95
LB3DC_ESTATE = -71
FP64 = 0
FP32_DEV = 1

DUMP_FIELDS = {"od": 1, "wd": 1, "sur": 1, "dir": 3, "vel": 1, "arr": 3, "rock": 1}

_D = ctypes.POINTER(ctypes.c_double)
_lib = None


class Lb3dError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"lb3dc error {code}: {msg}")
        self.code = code


def lib():
    """Loads liblb3dc.so; raises if the CUDA extension has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"CUDA extension {LIB_PATH} is missing: build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (needs nvcc)")
    L = ctypes.CDLL(LIB_PATH)
    H = ctypes.c_void_p
    I, LL, Dd = ctypes.c_int, ctypes.c_longlong, ctypes.c_double
    P = ctypes.POINTER(CParams)
    sigs = {
        "lb3dc_create": (I, [P, ctypes.POINTER(H)]),
        "lb3dc_destroy": (I, [H]),
        "lb3dc_last_error": (I, [H, ctypes.c_char_p, I]),
        "lb3dc_device_bytes": (LL, [H]),
        "lb3dc_footprint": (LL, [P]),
        "lb3dc_upload_state": (I, [H, _D, _D, _D, Dd, I]),
        "lb3dc_download_state": (I, [H, _D, _D, _D, _D, _D]),
        "lb3dc_upload_sites": (I, [H, _D, Dd, I]),
        "lb3dc_download_sites": (I, [H, _D]),
        "lb3dc_force_apply": (I, [H, I]),
        "lb3dc_bc_apply": (I, [H, I]),
        "lb3dc_advection": (I, [H]),
        "lb3dc_collision": (I, [H]),
        "lb3dc_time_loop": (I, [H, I]),
        "lb3dc_sync": (I, [H]),
        "lb3dc_set_launch_shape": (I, [H, I, I, I, I]),
        "lb3dc_get_launch_shape": (I, [H, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I),
                                       ctypes.POINTER(I)]),
        "lb3dc_autotune": (I, [H, _D, ctypes.POINTER(I)]),
        "lb3dc_stream": (ctypes.c_void_p, [H]),
        "lb3dc_set_profiling": (I, [H, I]),
        "lb3dc_kernel_stats": (I, [H, _D, ctypes.POINTER(LL), ctypes.POINTER(LL)]),
        "lb3dc_set_lees_edwards": (I, [H, Dd, Dd]),
        "lb3dc_get_lees_edwards": (I, [H, _D, _D]),
        "lb3dc_get_timestep": (I, [H, ctypes.POINTER(I)]),
        "lb3dc_reduce_conservation": (I, [H, _D, _D]),
        "lb3dc_sanity": (I, [H, ctypes.POINTER(LL), ctypes.POINTER(LL)]),
        "lb3dc_sanity_velocity": (I, [H, _D, ctypes.POINTER(I), _D, ctypes.POINTER(LL), ctypes.POINTER(LL)]),
        "lb3dc_dump": (I, [H, ctypes.c_char_p, _D]),
        "lb3dc_checkpoint_async": (I, [H, ctypes.c_char_p]),
        "lb3dc_dump_async": (I, [H, ctypes.c_char_p, ctypes.c_char_p, I]),
        "lb3dc_io_wait": (I, [H]),
        "lb3dc_xdr_read_checkpoint": (I, [ctypes.c_char_p, I, I, I, I, _D, _D, _D]),
        "lb3dc_xdr_write_checkpoint": (I, [ctypes.c_char_p, I, I, I, I, _D, _D, _D, _D]),
        "lb3dc_xdr_read_topo": (I, [ctypes.c_char_p, _D]),
        "lb3dc_xdr_write_topo": (I, [ctypes.c_char_p, Dd]),
        "lb3dc_xdr_read_rock": (I, [ctypes.c_char_p, I, I, I, _D]),
        "lb3dc_xdr_write_rock": (I, [ctypes.c_char_p, I, I, I, _D]),
        "lb3dc_xdr_write_field": (I, [ctypes.c_char_p, _D, LL, I, I]),
        "lb3dc_detmath_eval": (I, [I, I, _D, _D, LL]),
        "lb3dc_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_D)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Lattice:
    """One lattice resident on the current CUDA device."""

    def __init__(self, params: Params, precision: Optional[int] = None):
        p = params
        if precision is not None:
            p = Params(**{**p.__dict__, "precision": precision})
        p.validate()
        self.params = p
        self._cp = to_cparams(p)
        h = ctypes.c_void_p()
        rc = lib().lb3dc_create(ctypes.byref(self._cp), ctypes.byref(h))
        if rc != 0:
            raise Lb3dError(rc, self._error(None))
        self.h = h

    # -- errors -----------------------------------------------------------
    def _error(self, h):
        buf = ctypes.create_string_buffer(512)
        lib().lb3dc_last_error(h, buf, 512)
        return buf.value.decode(errors="replace")

    def _ck(self, rc):
        if rc != 0:
            raise Lb3dError(rc, self._error(self.h))
        return rc

    def close(self):
        if getattr(self, "h", None):
            lib().lb3dc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- geometry ---------------------------------------------------------
    @property
    def shape(self):
        return (self.params.nz, self.params.ny, self.params.nx)

    @property
    def nsites(self):
        return self.params.nx * self.params.ny * self.params.nz

    @property
    def device_bytes(self):
        return int(lib().lb3dc_device_bytes(self.h))

    # -- state ------------------------------------------------------------
    def upload(self, n, db=None, rock=None, shear_sum=0.0, nt=0):
        n, db, rock = _f64(n), _f64(db), _f64(rock)
        self._keep = (n, db, rock)
        self._ck(lib().lb3dc_upload_state(self.h, ptr(n), ptr(db), ptr(rock), float(shear_sum), int(nt)))

    def upload_state(self, state):
        self.upload(state["n"], state.get("db"), state.get("rock"), state.get("shear_sum", 0.0),
                    state.get("nt0", 0))

    def download(self):
        nc = self.params.ncomp
        sh = self.shape
        out = dict(n=np.empty((nc, 19) + sh), db=np.empty((3,) + sh), rho=np.empty((nc,) + sh),
                   mom=np.empty((nc, 3) + sh), da=np.empty((3,) + sh))
        self._ck(lib().lb3dc_download_state(self.h, ptr(out["n"]), ptr(out["db"]), ptr(out["rho"]),
                                            ptr(out["mom"]), ptr(out["da"])))
        return out

    def upload_sites(self, whole_n, shear_sum=0.0, nt=0):
        w = _f64(whole_n)
        self._ck(lib().lb3dc_upload_sites(self.h, ptr(w), float(shear_sum), int(nt)))

    def download_sites(self):
        sd = 79 if self.params.ncomp == 3 else 49
        p = self.params
        w = np.zeros((p.nz + 2, p.ny + 2, p.nx + 2, sd))
        self._ck(lib().lb3dc_download_sites(self.h, ptr(w)))
        return w

    # -- the time-loop stages (code/lb3d_time_loop.F90:58-92) ---------------
    def force_apply(self, stage):
        self._ck(lib().lb3dc_force_apply(self.h, int(stage)))

    def bc_apply(self, stage):
        self._ck(lib().lb3dc_bc_apply(self.h, int(stage)))

    def advection(self):
        self._ck(lib().lb3dc_advection(self.h))

    def collision(self):
        self._ck(lib().lb3dc_collision(self.h))

    def time_loop(self, nsteps):
        self._ck(lib().lb3dc_time_loop(self.h, int(nsteps)))

    def sync(self):
        self._ck(lib().lb3dc_sync(self.h))

    # -- FP32 launch shape ------------------------------------------------
    def set_launch_shape(self, tx, ty, zc, split=0):
        self._ck(lib().lb3dc_set_launch_shape(self.h, int(tx), int(ty), int(zc), int(split)))

    @property
    def launch_shape(self):
        a, b, c, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._ck(lib().lb3dc_get_launch_shape(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                              ctypes.byref(d)))
        return a.value, b.value, c.value, d.value

    def autotune(self):
        ms = np.zeros(64)
        n = ctypes.c_int()
        self._ck(lib().lb3dc_autotune(self.h, ptr(ms), ctypes.byref(n)))
        return self.launch_shape, ms[: n.value].tolist()

    # -- measurement ------------------------------------------------------
    @property
    def stream(self):
        return lib().lb3dc_stream(self.h)

    def set_profiling(self, on=True):
        self._ck(lib().lb3dc_set_profiling(self.h, int(bool(on))))

    def kernel_stats(self):
        """(device ms of the bracketed dominant kernels, their launch count,
        all kernel launches issued) since set_profiling."""
        ms = ctypes.c_double()
        n, alln = ctypes.c_longlong(), ctypes.c_longlong()
        self._ck(lib().lb3dc_kernel_stats(self.h, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(alln)))
        return ms.value, n.value, alln.value

    @property
    def timestep(self):
        v = ctypes.c_int()
        self._ck(lib().lb3dc_get_timestep(self.h, ctypes.byref(v)))
        return v.value

    @property
    def lees_edwards(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._ck(lib().lb3dc_get_lees_edwards(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    # -- observability ----------------------------------------------------
    def dump(self, field):
        k = DUMP_FIELDS[field]
        out = np.empty(self.nsites * k)
        self._ck(lib().lb3dc_dump(self.h, field.encode(), ptr(out)))
        return out

    def checkpoint_async(self, path):
        """Starts writing the current state as an XDR checkpoint file; the
        lattice may keep stepping.  io_wait() reports the outcome."""
        self._ck(lib().lb3dc_checkpoint_async(self.h, str(path).encode()))

    def dump_async(self, field, path, dump_double=False):
        self._ck(lib().lb3dc_dump_async(self.h, field.encode(), str(path).encode(), int(bool(dump_double))))

    def io_wait(self):
        self._ck(lib().lb3dc_io_wait(self.h))

    def conservation(self):
        m, u = np.zeros(3), np.zeros(3)
        self._ck(lib().lb3dc_reduce_conservation(self.h, ptr(m), ptr(u)))
        return m, u

    def sanity(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        rc = lib().lb3dc_sanity(self.h, ctypes.byref(a), ctypes.byref(b))
        if rc not in (0, LB3DC_ENAN):
            self._ck(rc)
        return a.value, b.value


    def sanity_velocity(self):
        """lbe_sanity_check's velocity statistics: dict with maxvel [species][axis],
        maxpos [species][axis][xyz] (1-based), velsum [species][axis], n_fluid,
        n_too_fast (sites with some species' |v| > 0.1)."""
        return _sanity_velocity(lib().lb3dc_sanity_velocity, self.h, self._ck)


def _sanity_velocity(fn, h, check):
    mv, vs = np.zeros(9), np.zeros(9)
    mp = (ctypes.c_int * 27)()
    nf, nt = ctypes.c_longlong(), ctypes.c_longlong()
    check(fn(h, ptr(mv), mp, ptr(vs), ctypes.byref(nf), ctypes.byref(nt)))
    return dict(maxvel=mv.reshape(3, 3), maxpos=np.array(mp[:], dtype=np.int64).reshape(3, 3, 3),
                velsum=vs.reshape(3, 3), n_fluid=nf.value, n_too_fast=nt.value)


def footprint(params: Params) -> int:
    cp = to_cparams(params)
    return int(lib().lb3dc_footprint(ctypes.byref(cp)))


# -- XDR files ---------------------------------------------------------------
def read_checkpoint(path, nx, ny, nz, ncomp):
    N = nx * ny * nz
    n = np.empty((ncomp, 19, nz, ny, nx))
    db = np.empty((3, nz, ny, nx)) if ncomp == 3 else None
    rock = np.empty((nz, ny, nx))
    rc = lib().lb3dc_xdr_read_checkpoint(path.encode(), nx, ny, nz, ncomp, ptr(n), ptr(db), ptr(rock))
    if rc != 0:
        raise Lb3dError(rc, f"cannot read checkpoint {path}")
    return dict(n=n, db=db, rock=rock)


def write_checkpoint(path, n, db=None, rock=None, da=None):
    n = _f64(n)
    ncomp, _, nz, ny, nx = n.shape
    da, db, rock = _f64(da), _f64(db), _f64(rock)
    rc = lib().lb3dc_xdr_write_checkpoint(path.encode(), nx, ny, nz, ncomp, ptr(n), ptr(da), ptr(db), ptr(rock))
    if rc != 0:
        raise Lb3dError(rc, f"cannot write checkpoint {path}")


def read_topo(path):
    v = ctypes.c_double()
    rc = lib().lb3dc_xdr_read_topo(path.encode(), ctypes.byref(v))
    if rc != 0:
        raise Lb3dError(rc, f"cannot read {path}")
    return v.value


def write_topo(path, shear_sum):
    rc = lib().lb3dc_xdr_write_topo(path.encode(), float(shear_sum))
    if rc != 0:
        raise Lb3dError(rc, f"cannot write {path}")


def read_rock(path, nx, ny, nz):
    rock = np.empty((nz, ny, nx))
    rc = lib().lb3dc_xdr_read_rock(path.encode(), nx, ny, nz, ptr(rock))
    if rc != 0:
        raise Lb3dError(rc, f"cannot read rock file {path}")
    return rock


def write_rock(path, rock):
    rock = _f64(rock)
    nz, ny, nx = rock.shape
    rc = lib().lb3dc_xdr_write_rock(path.encode(), nx, ny, nz, ptr(rock))
    if rc != 0:
        raise Lb3dError(rc, f"cannot write rock file {path}")


def write_field(path, values, values_per_site=1, dump_double=False):
    v = _f64(np.asarray(values).reshape(-1))
    nsites = v.size // values_per_site
    rc = lib().lb3dc_xdr_write_field(path.encode(), ptr(v), nsites, values_per_site, int(bool(dump_double)))
    if rc != 0:
        raise Lb3dError(rc, f"cannot write {path}")


def detmath_eval(fn, x, device=False):
    x = _f64(x)
    y = np.empty_like(x)
    rc = lib().lb3dc_detmath_eval({"exp": 0, "expm1": 1, "tanh": 2}[fn], int(device), ptr(x), ptr(y), x.size)
    if rc != 0:
        raise Lb3dError(rc, "detmath_eval failed")
    return y
