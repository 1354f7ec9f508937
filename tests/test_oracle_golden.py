"""Pins the CPU oracle against the reference's own golden vectors.

testLB3D.sh:280-300 runs each test of test/<T>/ for 10 steps from its t=0
checkpoint and byte-compares the FP32 XDR dumps with reference/*-t00000010.
The oracle is required to reproduce every golden value exactly (0 FP32
ulp), with glibc's exp/tanh and with the deterministic exp/tanh that the
device FP64 path uses."""
import numpy as np
import pytest

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
