"""Runs one synthetic lattice through the hot path and prints its step rate.

    python -m lb3d_b200.run_case --ncomp 3 --size 128 --precision fp32 \
        --shape 16,8,8,1 --steps 4 [--warmup 0] [--porosity 0.4] [--shear-u 0.05]

The state is the seeded uniform mixture (rho 0.7 + U(-0.01, 0.01) per
component, unit dipoles for ternary), or for --porosity the binary invasion
state in a seeded sphere pack with body force g_accn_x = 1e-5.  --shape
fixes the FP32 launch shape (tx, ty, z-chunk, split); "auto" runs the
autotuner.  The run is short and holds one lattice on the device, which is
what a profiler capture of a single kernel wants.
"""
from __future__ import annotations

import argparse
import json
import time

from .config import Params
from .ic import invasion_state, sphere_pack, uniform_mixture
from .lib import Lattice

PHYS = dict(tau_d=1.0, g_br=0.08, g_bs=-0.006, g_ss=-0.0045, beta=10.0, d_0=1.0, bdist=2, restore=1)


def make_case(ncomp, nx, ny, nz, precision, porosity=None, shear_u=0.0, seed=1):
    kw = dict(PHYS)
    if ncomp == 2:
        kw.pop("g_bs"), kw.pop("g_ss")
    if shear_u:
        kw.update(boundary_cond=-1, inv_fluid=5, shear_u=shear_u)
    if porosity is not None:
        kw.update(g_accn_x=1e-5)
    p = Params(nx=nx, ny=ny, nz=nz, ncomp=ncomp, precision=precision, **kw).finalize()
    if porosity is not None:
        rock = sphere_pack(nx, ny, nz, seed=seed, porosity=porosity, overlap=True)
        state = invasion_state(nx, ny, nz, rock, seed=seed)
    else:
        state = uniform_mixture(nx, ny, nz, ncomp, seed=seed)
    return p, state


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--ncomp", type=int, default=3, choices=[2, 3])
    ap.add_argument("--size", default="128", help="L or NXxNYxNZ")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--shape", default="auto", help="tx,ty,zc,split or auto (FP32 only)")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=0)
    ap.add_argument("--porosity", type=float, default=None)
    ap.add_argument("--shear-u", type=float, default=0.0)
    a = ap.parse_args(argv)
    dims = [int(v) for v in a.size.lower().split("x")]
    nx, ny, nz = dims if len(dims) == 3 else dims * 3
    prec = 1 if a.precision == "fp32" else 0
    p, state = make_case(a.ncomp, nx, ny, nz, prec, a.porosity, a.shear_u)
    lat = Lattice(p, precision=prec)
    lat.upload_state(state)
    if prec == 1:
        if a.shape == "auto":
            lat.autotune()
        else:
            lat.set_launch_shape(*[int(v) for v in a.shape.split(",")])
    if a.warmup:
        lat.time_loop(a.warmup)
    lat.sync()
    lat.set_profiling(True)
    t0 = time.perf_counter()
    lat.time_loop(a.steps)
    lat.sync()
    dt = time.perf_counter() - t0
    kms, nlaunch, _ = lat.kernel_stats()
    lat.set_profiling(False)
    mass, _ = lat.conservation()
    sites = nx * ny * nz
    print(json.dumps(dict(ncomp=a.ncomp, size=[nx, ny, nz], precision=a.precision,
                          shape=list(lat.launch_shape) if prec == 1 else None, steps=a.steps,
                          wall_mlups=round(sites * a.steps / dt / 1e6, 1),
                          device_ms_per_step=round(kms / max(nlaunch, 1), 4),
                          device_mlups=round(sites * nlaunch / max(kms, 1e-9) / 1e3, 1),
                          mass=[float(m) for m in mass[: a.ncomp]])))


if __name__ == "__main__":
    main()
