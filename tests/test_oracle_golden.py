"""Pins the CPU oracle against the reference's own golden vectors.

testLB3D.sh:280-300 runs each test of test/<T>/ for 10 steps from its t=0
checkpoint and byte-compares the FP32 XDR dumps with reference/*-t00000010.
The oracle is required to reproduce every golden value exactly (0 FP32
ulp), with glibc's exp/tanh and with the deterministic exp/tanh that the
device FP64 path uses."""
import numpy as np
import pytest

from lb3d_b200.config import Params
from tests._fixtures import CASES, FIELDS, load_case, load_golden
from tests._oracle import Oracle, set_math


def ulp_diff(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


@pytest.fixture(scope="module", params=[0, 1], ids=["libm", "detmath"])
def math_mode(request):
    set_math(request.param)
    yield request.param
    set_math(0)


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_reproduces_goldens(case, math_mode):
    p, st = load_case(case)
    o = Oracle(p, st)
    o.run(10)
    for field in FIELDS[case]:
        gold = load_golden(case, field)
        mine = o.dump(field).astype(np.float32)
        assert mine.shape == gold.shape
        u = ulp_diff(mine, gold)
        assert u.max() == 0, f"{case}/{field}: max {u.max()} ulp at {np.argmax(u)}"


def test_lees_edwards_shear_sum_bookkeeping():
    """The checktopo shear_sum 0.0106667 = 0.01*16/15 is reduced by one shear_u
    at init (code/lb3d_bc.F90:62-72) and increased by shear_u every stage 6."""
    p, st = load_case("leesEdwards")
    o = Oracle(p, st)
    su = 0.01 * 16.0 / 15.0
    assert abs(o.shear_sum - st["shear_sum"]) < 1e-15
    o.run(10)
    assert abs(o.shear_sum - (st["shear_sum"] + 10 * su)) < 1e-14


def test_rejects_fatal_combinations():
    p, st = load_case("gyroid")
    p.boundary_cond, p.inv_fluid = -1, 5  # ternary + Lees-Edwards is fatal
    with pytest.raises(ValueError):
        Oracle(p, st)


@pytest.mark.parametrize("inv_fluid", [7, 8])
def test_recolouring_stage(inv_fluid):
    """lbe_invade_binary (code/lb3d_invasion.F90:1257-1358) at stage 8: the
    two bottom planes carry all of n_r + n_b as red (inv_fluid 7) or blue
    (8), the two top planes the other colour; rock sites and the planes in
    between are untouched, and every population's n_r + n_b is kept."""
    from lb3d_b200.ic import uniform_mixture
    dims = (8, 6, 7)
    p = Params(nx=8, ny=6, nz=7, ncomp=2, bdist=2, boundary_cond=-1, inv_fluid=inv_fluid,
               g_br=0.08).finalize()
    st = uniform_mixture(*dims, 2, seed=3)
    rock = np.zeros((7, 6, 8))
    rock[1, 2, 3] = 1.0
    rock[5, 4, 0] = 1.0
    st["rock"] = rock
    o = Oracle(p, st)
    o.stage(6)
    o.stage(7)
    before = o.get()["n"]
    o.stage(8)
    after = o.get()["n"]
    fill, empty = (0, 1) if inv_fluid == 7 else (1, 0)
    fluid = rock == 0
    tot = before[0] + before[1]
    for z in (0, 1):
        m = fluid[z]
        assert np.all(after[empty][:, z][:, m] == 0.0)
        np.testing.assert_array_equal(after[fill][:, z][:, m], tot[:, z][:, m])
    for z in (5, 6):
        m = fluid[z]
        assert np.all(after[fill][:, z][:, m] == 0.0)
        np.testing.assert_array_equal(after[empty][:, z][:, m], tot[:, z][:, m])
    np.testing.assert_array_equal(after[:, :, 2:5], before[:, :, 2:5])
    np.testing.assert_array_equal(after[:, :, 1, 2, 3], before[:, :, 1, 2, 3])
    np.testing.assert_array_equal(after[:, :, 5, 4, 0], before[:, :, 5, 4, 0])


def test_recolouring_is_binary_only():
    from lb3d_b200.ic import uniform_mixture
    p = Params(nx=6, ny=6, nz=6, ncomp=3, bdist=2, boundary_cond=-1, inv_fluid=7).finalize()
    with pytest.raises(ValueError):
        p.validate()
    with pytest.raises(ValueError):
        Oracle(p, uniform_mixture(6, 6, 6, 3, seed=1))


def test_zouhe_density_stage_sets_boundary_densities():
    """lbe_invade_zouandhe (code/lb3d_invasion.F90:1459-1796) at stage 8:
    the red and blue densities of the fluid sites of z = 1 become fr, fb
    and those of z = nz become pr, pb (the closure conserves the density it
    is given; equal masses here), the planes in between are untouched."""
    from lb3d_b200.ic import uniform_mixture
    p = Params(nx=7, ny=6, nz=5, ncomp=2, bdist=2, boundary_cond=-1, inv_fluid=11, g_br=0.08,
               fr=0.8, fb=0.6, pr=0.65, pb=0.75).finalize()
    st = uniform_mixture(7, 6, 5, 2, seed=4)
    o = Oracle(p, st)
    o.stage(6)
    o.stage(7)
    before = o.get()["n"]
    o.stage(8)
    after = o.get()["n"]
    g = np.array([2.0] * 6 + [1.0] * 12 + [1.0])  # reference weights: axes 2, rest 1
    rho = np.einsum("cqzyx,q->czyx", after, g)
    np.testing.assert_allclose(rho[0, 0], 0.8, rtol=0, atol=1e-14)
    np.testing.assert_allclose(rho[1, 0], 0.6, rtol=0, atol=1e-14)
    np.testing.assert_allclose(rho[0, 4], 0.65, rtol=0, atol=1e-14)
    np.testing.assert_allclose(rho[1, 4], 0.75, rtol=0, atol=1e-14)
    np.testing.assert_array_equal(after[:, :, 1:4], before[:, :, 1:4])
