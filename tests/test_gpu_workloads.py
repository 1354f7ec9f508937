"""Parity at the benchmark workloads' own sizes.

The throughput figures are quoted on three single-lattice workloads; each
runs here through the product path and through the CPU oracle (OpenMP, all
host threads) from the same seeded state:

* ternary amphiphilic 128^3, periodic (g_br 0.08, g_bs -0.006, g_ss -0.0045);
* binary Lees-Edwards 256x128x128, x-planes sheared at shear_u 0.05;
* binary invasion through porous rock 256^3 (overlapping spheres of radius
  6..12 at porosity 0.4, body force 1e-5 along x, red inlet slab).

The FP64 drop-in path must equal the oracle bit for bit (the oracle runs the
device's deterministic exp/tanh).  The FP32 deviation path runs the launch
shape its autotuner picks for the lattice -- the shape the benchmark uses --
and must stay within the FP32 tolerances of tests/test_gpu_fp32.py.  These
sizes exercise what small lattices cannot: 32-bit offsets over millions of
sites, full tiles and z chunks at 128 and 256, the narrow-offset moments
pass and the porous lattice's tuned shape."""
import numpy as np
import pytest

from lb3d_b200.config import Params
from lb3d_b200.ic import invasion_state, sphere_pack, uniform_mixture
from tests._oracle import Oracle, set_math

pytestmark = pytest.mark.gpu
RHO_ATOL, DB_ATOL, N_ATOL = 1e-5, 2e-4, 2e-6
PHYS = dict(tau_d=1.0, beta=10.0, d_0=1.0, bdist=2, restore=1, g_br=0.08)


def ternary_128():
    p = Params(nx=128, ny=128, nz=128, ncomp=3, g_bs=-0.006, g_ss=-0.0045, **PHYS).finalize()
    return p, uniform_mixture(128, 128, 128, 3, seed=1)


def lees_edwards_256():
    p = Params(nx=256, ny=128, nz=128, ncomp=2, boundary_cond=-1, inv_fluid=5, shear_u=0.05,
               **PHYS).finalize()
    return p, uniform_mixture(256, 128, 128, 2, seed=3)


def porous_256():
    rock = sphere_pack(256, 256, 256, seed=4, porosity=0.4, rmin=6, rmax=12, overlap=True)
    p = Params(nx=256, ny=256, nz=256, ncomp=2, g_accn_x=1e-5, **PHYS).finalize()
    return p, invasion_state(256, 256, 256, rock, seed=4)


WORKLOADS = {"ternary-128": (ternary_128, 20), "lees-edwards-256x128x128": (lees_edwards_256, 10),
             "porous-256": (porous_256, 5)}


def _run_oracle(p, st, steps):
    set_math(1)
    try:
        o = Oracle(p, st)
        o.run(steps)
        return o.get(), o
    finally:
        set_math(0)


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_fp64_bit_identical_at_workload_size(name):
    from lb3d_b200.lib import Lattice
    make, steps = WORKLOADS[name]
    p, st = make()
    lat = Lattice(p, precision=0)
    lat.upload_state(st)
    lat.time_loop(steps)
    a = lat.download()
    shear_sum = lat.lees_edwards[0] if p.lees_edwards else None
    lat.close()
    b, o = _run_oracle(p, st, steps)
    for k in ("n", "rho", "mom"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{name} {k}")
    if p.ncomp == 3:
        np.testing.assert_array_equal(a["db"], b["db"], err_msg=f"{name} db")
        np.testing.assert_array_equal(a["da"], b["da"], err_msg=f"{name} da")
    if p.lees_edwards:
        assert shear_sum == o.shear_sum


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_fp32_within_tolerance_at_workload_size(name):
    from lb3d_b200.lib import Lattice
    make, steps = WORKLOADS[name]
    p, st = make()
    lat = Lattice(p, precision=1)
    lat.upload_state(st)
    shape, _ = lat.autotune()  # restores the uploaded state after timing
    lat.time_loop(steps)
    a = lat.download()
    lat.close()
    b, _ = _run_oracle(p, st, steps)
    err = np.abs(a["rho"] - b["rho"]).max()
    assert err <= RHO_ATOL, f"{name} {shape}: rho err {err:.3e}"
    err = np.abs(a["n"] - b["n"]).max()
    assert err <= N_ATOL, f"{name} {shape}: n err {err:.3e}"
    if p.ncomp == 3:
        err = np.abs(a["db"] - b["db"]).max()
        assert err <= DB_ATOL, f"{name} {shape}: db err {err:.3e}"
