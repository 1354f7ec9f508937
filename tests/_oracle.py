"""ctypes binding of the CPU oracle (oracle/lb3d_oracle.h).  Test
infrastructure: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py."""
import ctypes
import os

import numpy as np

from lb3d_b200.config import _C_FIELDS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "_build", "liblb3d_oracle.so")


class OParams(ctypes.Structure):
    _fields_ = list(_C_FIELDS)


_lib = None
HALO_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        D, I, V = ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_void_p
        L.lb3do_create.restype = V
        L.lb3do_create.argtypes = [ctypes.POINTER(OParams)]
        L.lb3do_destroy.argtypes = [V]
        L.lb3do_set_threads.argtypes = [I]
        L.lb3do_set_math.argtypes = [I]
        L.lb3do_load.argtypes = [V, D, D, D, ctypes.c_double, I]
        L.lb3do_stage.argtypes = [V, I]
        L.lb3do_run.argtypes = [V, I]
        L.lb3do_get.argtypes = [V, D, D, D, D, D]
        L.lb3do_dump.argtypes = [V, ctypes.c_char_p, D]
        L.lb3do_sums.argtypes = [V, D, D]
        L.lb3do_sanity_velocity.argtypes = [V, D, ctypes.POINTER(ctypes.c_int), D,
                                            ctypes.POINTER(ctypes.c_longlong),
                                            ctypes.POINTER(ctypes.c_longlong)]
        L.lb3do_set_slab.argtypes = [V, I, HALO_FN, V]
        L.lb3do_yplane_doubles.argtypes = [V]
        L.lb3do_yplane_doubles.restype = ctypes.c_longlong
        L.lb3do_yplane.argtypes = [V, I, D, I]
        L.lb3do_shear_sum.argtypes = [V]
        L.lb3do_shear_sum.restype = ctypes.c_double
        L.lb3do_nt.argtypes = [V]
        _lib = L
    return _lib


def set_math(det):
    """0: glibc exp/tanh; 1: the deterministic exp/tanh of the device FP64 path."""
    lib().lb3do_set_math(int(det))


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """One reference-equivalent lattice on the CPU."""

    def __init__(self, p, state, threads=0, slab=None):
        """slab = (y_off, exchange): this oracle holds p.ny planes of a
        lattice split along y, starting at global plane y_off (p carries the
        global-coordinate parameters); exchange(oracle) fills its y-halo
        planes from the neighbouring slabs at every halo exchange."""
        L = lib()
        if threads:
            L.lb3do_set_threads(threads)
        c = OParams()
        for name, _ in OParams._fields_:
            setattr(c, name, getattr(p, name))
        self.h = L.lb3do_create(ctypes.byref(c))
        if not self.h:
            raise ValueError("oracle rejected the parameter set")
        self.p = p
        if slab is not None:
            y_off, exchange = slab
            self._hook = HALO_FN(lambda ctx, h: exchange(self))
            if L.lb3do_set_slab(self.h, int(y_off), self._hook, None) != 0:
                raise ValueError("slab rejected")
        n = np.ascontiguousarray(state["n"], dtype=np.float64)
        db = state.get("db")
        db = None if db is None else np.ascontiguousarray(db, dtype=np.float64)
        rock = state.get("rock")
        rock = None if rock is None else np.ascontiguousarray(rock, dtype=np.float64)
        self._keep = (n, db, rock)
        L.lb3do_load(self.h, _ptr(n), _ptr(db), _ptr(rock), float(state.get("shear_sum", 0.0)),
                     int(state.get("nt0", 0)))

    def __del__(self):
        if getattr(self, "h", None):
            lib().lb3do_destroy(self.h)
            self.h = None

    def run(self, nsteps):
        lib().lb3do_run(self.h, int(nsteps))

    def stage(self, s):
        if lib().lb3do_stage(self.h, int(s)) != 0:
            raise ValueError(s)

    @property
    def shape(self):
        return (self.p.nz, self.p.ny, self.p.nx)

    def get(self):
        nc = self.p.ncomp
        sh = self.shape
        n = np.empty((nc, 19) + sh)
        db = np.empty((3,) + sh)
        rho = np.empty((nc,) + sh)
        mom = np.empty((nc, 3) + sh)
        da = np.empty((3,) + sh)
        lib().lb3do_get(self.h, _ptr(n), _ptr(db), _ptr(rho), _ptr(mom), _ptr(da))
        return dict(n=n, db=db, rho=rho, mom=mom, da=da)

    def dump(self, field):
        sh = self.shape
        k = 3 if field in ("dir", "arr") else 1
        out = np.empty(int(np.prod(sh)) * k)
        if lib().lb3do_dump(self.h, field.encode(), _ptr(out)) != 0:
            raise ValueError(field)
        return out

    def yplane(self, y):
        """Whole sites of plane y (0 .. ny + 1), x = 0..nx+1, z = 1..nz, as doubles."""
        out = np.empty(lib().lb3do_yplane_doubles(self.h))
        lib().lb3do_yplane(self.h, int(y), _ptr(out), 0)
        return out

    def set_yplane(self, y, buf):
        buf = np.ascontiguousarray(buf, dtype=np.float64)
        lib().lb3do_yplane(self.h, int(y), _ptr(buf), 1)

    def sums(self):
        m = np.zeros(3)
        u = np.zeros(3)
        lib().lb3do_sums(self.h, _ptr(m), _ptr(u))
        return m, u

    def sanity_velocity(self):
        from lb3d_b200.lib import _sanity_velocity
        return _sanity_velocity(lib().lb3do_sanity_velocity, self.h, lambda rc: None)

    @property
    def shear_sum(self):
        return lib().lb3do_shear_sum(self.h)
