"""Ensembles of independent lattices and the serving loop over them.

`Ensemble` wraps the lb3dc_ensemble_* C-ABI: members of uneven size share
one packed, device-resident site space and advance together in one
persistent fused kernel launch per step (replayed from a CUDA graph).

`Server` is the request loop for parameter-sweep solves: requests that have
arrived are admitted in arrival order while their HBM footprint fits in the
ensemble's free site space (first-fit ranges), all admitted requests advance
together, and finished ones are retired (result downloaded, space freed)
as soon as they complete, so later arrivals join while earlier ones are
still running (continuous batching).  It reports throughput (solves/s) and
time-to-result percentiles.
"""
from __future__ import annotations

import ctypes
import dataclasses
import time
from typing import Dict, List, Optional

import numpy as np

from .config import CParams, Params, to_cparams
from .lib import LB3DC_ENOMEM, Lb3dError, lib, ptr

_D = ctypes.POINTER(ctypes.c_double)


def _bind():
    L = lib()
    if getattr(L, "_ens_bound", False):
        return L
    V, I, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
    P = ctypes.POINTER(CParams)
    sigs = {
        "lb3dc_ensemble_create": (I, [I, LL, I, ctypes.POINTER(V)]),
        "lb3dc_ensemble_destroy": (I, [V]),
        "lb3dc_ensemble_last_error": (I, [V, ctypes.c_char_p, I]),
        "lb3dc_ensemble_set_shape": (I, [V, I, I, I, I]),
        "lb3dc_ensemble_admit": (I, [V, P, _D, _D, I, ctypes.POINTER(I)]),
        "lb3dc_ensemble_admit_seeded": (I, [V, P, ctypes.c_ulonglong, _D, ctypes.c_double, I,
                                            ctypes.POINTER(I)]),
        "lb3dc_ensemble_step": (I, [V, I, ctypes.POINTER(I)]),
        "lb3dc_ensemble_sync": (I, [V]),
        "lb3dc_ensemble_finished": (I, [V, ctypes.POINTER(I), I, ctypes.POINTER(I)]),
        "lb3dc_ensemble_retire": (I, [V, I, _D, _D]),
        "lb3dc_ensemble_stats": (I, [V, ctypes.POINTER(LL), ctypes.POINTER(I), ctypes.POINTER(I),
                                     ctypes.POINTER(LL)]),
        "lb3dc_ensemble_bytes": (LL, [V]),
        "lb3dc_ensemble_retire_async": (I, [V, I, _D, _D]),
        "lb3dc_ensemble_poll": (I, [V, I, ctypes.POINTER(I)]),
        "lb3dc_host_alloc": (I, [LL, ctypes.POINTER(V)]),
        "lb3dc_host_free": (I, [V]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args
    L._ens_bound = True
    return L


def member_bytes(p: Params) -> int:
    """Device bytes one member occupies in an ensemble (FP32 deviations, two
    buffers, plus dipoles and the rock byte)."""
    n = p.nx * p.ny * p.nz
    return n * (2 * 19 * p.ncomp * 4 + (24 if p.ncomp == 3 else 0) + 1)


class PinnedPool:
    """Reusable page-locked host blocks (lb3dc_host_alloc) viewed as float64
    arrays; a block is taken for a shape and given back after use."""

    def __init__(self):
        self.free = []    # (capacity in elements, pointer)
        self.owned = {}   # id(array) -> (capacity, pointer)

    def take(self, shape):
        count = int(np.prod(shape))
        for k, (cap, p) in enumerate(self.free):
            if cap >= count:
                self.free.pop(k)
                break
        else:
            # idle blocks too small for this request go back to the system,
            # so a long stream of mixed sizes keeps the pool near its peak need
            small = [(c, q) for c, q in self.free if c < count]
            self.free = [(c, q) for c, q in self.free if c >= count]
            for _, q in small:
                _bind().lb3dc_host_free(ctypes.c_void_p(q))
            p = ctypes.c_void_p()
            rc = _bind().lb3dc_host_alloc(ctypes.c_longlong(count * 8), ctypes.byref(p))
            if rc != 0:
                raise Lb3dError(rc, "pinned host allocation failed")
            cap, p = count, p.value
        buf = (ctypes.c_double * cap).from_address(p)
        arr = np.ctypeslib.as_array(buf)[:count].reshape(shape)
        self.owned[id(arr)] = (cap, p)
        return arr

    def give(self, arr):
        self.free.append(self.owned.pop(id(arr)))

    def release(self):
        for cap, p in self.free + list(self.owned.values()):
            _bind().lb3dc_host_free(ctypes.c_void_p(p))
        self.free, self.owned = [], {}


class Ensemble:
    def __init__(self, ncomp=3, capacity_sites=1 << 24, max_lattices=1024, shape=(32, 4, 8, 2)):
        L = _bind()
        h = ctypes.c_void_p()
        rc = L.lb3dc_ensemble_create(int(ncomp), int(capacity_sites), int(max_lattices), ctypes.byref(h))
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            L.lb3dc_last_error(None, buf, 512)
            raise Lb3dError(rc, buf.value.decode())
        self.h = h
        self.ncomp = ncomp
        self.capacity = capacity_sites
        self._pinned = PinnedPool()
        self._pending = {}
        if shape:
            sh = tuple(shape) + ((1,) if len(shape) == 3 else ())
            self._ck(L.lb3dc_ensemble_set_shape(self.h, *map(int, sh)))

    def _err(self):
        buf = ctypes.create_string_buffer(512)
        _bind().lb3dc_ensemble_last_error(self.h, buf, 512)
        return buf.value.decode()

    def _ck(self, rc):
        if rc != 0:
            raise Lb3dError(rc, self._err())

    def close(self):
        if getattr(self, "h", None):
            _bind().lb3dc_ensemble_destroy(self.h)
            self.h = None
        if getattr(self, "_pinned", None):
            self._pinned.release()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, p: Params, state=None, steps=0, seed=None, rho=(0.7, 0.7, 0.7), amp=0.01):
        """Returns the member slot, or None when the ensemble has no room."""
        cp = to_cparams(p)
        slot = ctypes.c_int()
        if state is not None:
            n = np.ascontiguousarray(state["n"], dtype=np.float64)
            db = state.get("db")
            db = None if db is None else np.ascontiguousarray(db, dtype=np.float64)
            rc = _bind().lb3dc_ensemble_admit(self.h, ctypes.byref(cp), ptr(n), ptr(db), int(steps),
                                              ctypes.byref(slot))
        else:
            r = (ctypes.c_double * 3)(*rho)
            rc = _bind().lb3dc_ensemble_admit_seeded(self.h, ctypes.byref(cp), ctypes.c_ulonglong(seed or 1),
                                                     ctypes.cast(r, _D), float(amp), int(steps),
                                                     ctypes.byref(slot))
        if rc == LB3DC_ENOMEM:
            return None
        self._ck(rc)
        return slot.value

    def step(self, max_steps):
        done = ctypes.c_int()
        self._ck(_bind().lb3dc_ensemble_step(self.h, int(max_steps), ctypes.byref(done)))
        return done.value

    def sync(self):
        self._ck(_bind().lb3dc_ensemble_sync(self.h))

    def finished(self) -> List[int]:
        n = ctypes.c_int()
        _bind().lb3dc_ensemble_finished(self.h, None, 0, ctypes.byref(n))
        arr = (ctypes.c_int * max(1, n.value))()
        _bind().lb3dc_ensemble_finished(self.h, arr, n.value, ctypes.byref(n))
        return list(arr[: n.value])

    def retire(self, slot, shape=None, download=True):
        """Frees the member; returns its populations (and dipoles) when
        `download` and `shape` = (nz, ny, nx) are given."""
        out = None
        if download and shape is not None:
            n = np.empty((self.ncomp, 19) + tuple(shape))
            db = np.empty((3,) + tuple(shape)) if self.ncomp == 3 else None
            self._ck(_bind().lb3dc_ensemble_retire(self.h, int(slot), ptr(n), ptr(db)))
            out = dict(n=n, db=db)
        else:
            self._ck(_bind().lb3dc_ensemble_retire(self.h, int(slot), None, None))
        return out

    # -- asynchronous retire --------------------------------------------
    def retire_async(self, slot, shape):
        """Starts copying a finished member's populations (and dipoles) to
        pinned host buffers while the ensemble keeps stepping; `poll` tells
        when they have landed and `collect` returns them."""
        n = self._pinned.take((self.ncomp, 19) + tuple(shape))
        db = self._pinned.take((3,) + tuple(shape)) if self.ncomp == 3 else None
        self._ck(_bind().lb3dc_ensemble_retire_async(self.h, int(slot), ptr(n), ptr(db)))
        self._pending[slot] = (n, db)

    def poll(self, slot) -> bool:
        done = ctypes.c_int()
        self._ck(_bind().lb3dc_ensemble_poll(self.h, int(slot), ctypes.byref(done)))
        return bool(done.value)

    def collect(self, slot):
        """Copies a landed asynchronous retire out of the pinned buffers."""
        n, db = self._pending.pop(slot)
        out = dict(n=n.copy(), db=None if db is None else db.copy())
        self._pinned.give(n)
        if db is not None:
            self._pinned.give(db)
        return out

    def stats(self):
        fs, a, r, su = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        _bind().lb3dc_ensemble_stats(self.h, ctypes.byref(fs), ctypes.byref(a), ctypes.byref(r), ctypes.byref(su))
        return dict(free_sites=fs.value, active=a.value, resident=r.value, site_updates=su.value)


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float  # seconds after the start of the stream
    params: Params
    steps: int
    seed: int
    result: Optional[dict] = None
    admitted: Optional[float] = None
    done: Optional[float] = None


def sweep_requests(n, seed=7, rate=200.0, lmin=16, lmax=96, steps=(500, 5000), ncomp=3,
                   base: Optional[Params] = None) -> List[Request]:
    """Seeded parameter-sweep requests: Poisson arrivals (mean `rate` per s),
    cubic edges log-uniform in [lmin, lmax], g_br in [0.06, 0.10], g_bs in
    [-0.008, -0.002], g_ss in [-0.006, -0.003], steps uniform."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        L = int(round(np.exp(rng.uniform(np.log(lmin), np.log(lmax)))))
        g_br = rng.uniform(0.06, 0.10)
        g_bs = rng.uniform(-0.008, -0.002)
        g_ss = rng.uniform(-0.006, -0.003)
        nst = int(rng.integers(steps[0], steps[1] + 1))
        b = base or Params(tau_d=1.0, beta=10.0, d_0=1.0, bdist=2, restore=1)
        p = dataclasses.replace(b, nx=L, ny=L, nz=L, ncomp=ncomp, g_br=g_br, g_bs=g_bs, g_ss=g_ss,
                                precision=1).finalize()
        p.g_accn_max, p.g_accn_max_x, p.g_accn_max_y = L, L, L
        out.append(Request(i, t, p, nst, seed=1000 + i))
    return out


class Server:
    """Continuous-batching request loop over one Ensemble.  Finished members
    are retired asynchronously: their results travel to the host while the
    others step, and a request is done when its results have landed.

    on_result(request, result) receives each result as it lands, and the
    server keeps nothing of it (a long stream of large lattices would
    otherwise fill host memory); without a callback the result is kept on
    the request as `request.result`."""

    def __init__(self, ensemble: Ensemble, chunk=64, download=True, on_result=None):
        self.ens = ensemble
        self.chunk = chunk
        self.download = download
        self.on_result = on_result

    def _collect(self, copying, done, clock, wait=False):
        while copying:
            landed = [s for s in list(copying) if self.ens.poll(s)]
            for s in landed:
                r = copying.pop(s)
                res = self.ens.collect(s)
                r.done = clock()
                if self.on_result is not None:
                    self.on_result(r, res)
                else:
                    r.result = res
                done.append(r)
            if not wait or not copying:
                return
            time.sleep(0.0005)

    def run(self, requests: List[Request], realtime=True, time_scale=1.0):
        reqs = sorted(requests, key=lambda r: r.arrival)
        queue: List[Request] = []
        live: Dict[int, Request] = {}
        copying: Dict[int, Request] = {}  # finished, results on their way to the host
        nxt = 0
        t0 = time.perf_counter()
        clock = lambda: (time.perf_counter() - t0) / time_scale  # noqa: E731
        done = []
        while len(done) < len(reqs):
            now = clock() if realtime else float("inf")
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                queue.append(reqs[nxt])
                nxt += 1
            # admit in arrival order while the footprint fits
            while queue:
                r = queue[0]
                slot = self.ens.admit(r.params, steps=r.steps, seed=r.seed)
                if slot is None:
                    break
                r.admitted = clock()
                live[slot] = r
                queue.pop(0)
            if not live:
                if copying:
                    self._collect(copying, done, clock, wait=True)
                elif nxt < len(reqs) and realtime:
                    time.sleep(max(0.0, (reqs[nxt].arrival - clock()) * time_scale))
                continue
            self.ens.step(self.chunk)
            # while the GPU steps: hand over the results that have landed
            self._collect(copying, done, clock)
            self.ens.sync()
            for slot in self.ens.finished():
                r = live.pop(slot)
                if self.download:
                    self.ens.retire_async(slot, (r.params.nz, r.params.ny, r.params.nx))
                    copying[slot] = r
                else:
                    self.ens.retire(slot, download=False)
                    r.done = clock()
                    done.append(r)
            if not live and copying and not queue:
                self._collect(copying, done, clock, wait=True)
        self._collect(copying, done, clock, wait=True)
        wall = clock()
        lat = np.array([r.done - r.arrival for r in done])
        first = min(r.arrival for r in reqs)
        return dict(
            solves=len(done), wall_s=wall, solves_per_s=len(done) / max(wall - first, 1e-9),
            p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
            mean_s=float(lat.mean()),
            site_updates=int(sum(r.params.nx * r.params.ny * r.params.nz * r.steps for r in done)),
        )
