"""FP32 deviation path against the FP64 drop-in path after 10 000 steps.

The FP64 path equals the oracle bit for bit (tests/test_gpu_fp64_parity.py,
tests/test_gpu_workloads.py), so it stands in for the oracle here.

* Binary mixture below the spinodal (g_br 0.02, densities 0.7 each): the
  fluctuations of the seeded mixture decay and nothing amplifies a rounding
  difference, so the pointwise bound holds directly: max |drho| and
  max |dphi| (phi = rho_r - rho_b) at most 1e-5 after 10 000 steps.
* Ternary amphiphilic mixture at g_br 0.01 with the headline surfactant
  couplings (g_bs -0.006, g_ss -0.0045): the surfactant forms a pattern on
  the lattice scale, whose growth amplifies any difference, so the FP64
  path itself moves by ~2e-5 when its initial populations are perturbed by
  1e-7 relative.  Equal accuracy: the FP32 path's density, order-parameter
  and velocity differences stay within twice that FP64 response, and its
  order-parameter difference within 1e-5.
"""
import numpy as np
import pytest

from lb3d_b200.config import Params
from lb3d_b200.ic import uniform_mixture
from lb3d_b200.lib import Lattice

pytestmark = pytest.mark.gpu
STEPS = 10_000
PHYS = dict(tau_d=1.0, beta=10.0, d_0=1.0, bdist=2, restore=1)


# D3Q19 degeneracies and velocities in the reference's direction order
# (code/lb3d_lattice.F90:137-187); the populations carry the weights w_i / g_i
_G = np.array([2.0] * 6 + [1.0] * 13)
_C = np.array([[1, -1, 0, 0, 0, 0, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0, 0],
               [0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0],
               [0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, 0]], dtype=np.float64)


def _velocity(r):
    """Barycentric velocity of the current populations (the FP64 path's
    stored momenta are those of the last advection, before its collision)."""
    w = r["n"].sum(0) * _G[:, None, None, None]
    return np.tensordot(_C, w, axes=(1, 0)) / w.sum(0)[None]


def _diffs(r, ref):
    drho = np.abs(r["rho"] - ref["rho"]).max()
    dphi = np.abs((r["rho"][0] - r["rho"][1]) - (ref["rho"][0] - ref["rho"][1])).max()
    du = np.abs(_velocity(r) - _velocity(ref)).max()
    return drho, dphi, du


def _run(p, st, precision):
    lat = Lattice(p, precision=precision)
    try:
        lat.upload_state(st)
        if precision == 1:
            lat.autotune()
        lat.time_loop(STEPS)
        return lat.download()
    finally:
        lat.close()


def test_binary_below_spinodal_pointwise_1e5():
    p = Params(nx=64, ny=64, nz=64, ncomp=2, g_br=0.02, **PHYS).finalize()
    st = uniform_mixture(64, 64, 64, 2, seed=5)
    ref = _run(p, st, 0)
    r32 = _run(p, st, 1)
    drho, dphi, du = _diffs(r32, ref)
    assert drho <= 1e-5 and dphi <= 1e-5, (drho, dphi, du)


def test_ternary_mixed_within_fp64_sensitivity():
    p = Params(nx=64, ny=64, nz=64, ncomp=3, g_br=0.01, g_bs=-0.006, g_ss=-0.0045,
               **PHYS).finalize()
    st = uniform_mixture(64, 64, 64, 3, seed=2)
    pert = dict(st)
    rng = np.random.default_rng(99)
    pert["n"] = st["n"] * (1.0 + 1e-7 * (2.0 * rng.random(st["n"].shape) - 1.0))
    ref = _run(p, st, 0)
    floor = _diffs(_run(p, pert, 0), ref)
    got = _diffs(_run(p, st, 1), ref)
    assert got[1] <= 1e-5, (got, floor)
    for g, f in zip(got, floor):
        assert g <= 2.0 * f, (got, floor)
