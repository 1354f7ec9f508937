"""FP32 deviation-storage path (LB3DC_FP32_DEV) against the FP64 oracle.

The FP32 path stores n - w_i rho0 in FP32 and collides in FP32, so it is
compared with absolute tolerances (the deviation storage carries absolute,
not per-site relative, precision): after 20 steps of the reference's test
systems the densities must agree to 1e-5, the dipoles to 2e-4 and the
populations to 2e-6 (populations are ~0.02, densities ~0.7)."""
import numpy as np
import pytest

from lb3d_b200.config import Params
from lb3d_b200.ic import uniform_mixture
from tests._fixtures import load_case
from tests._oracle import Oracle, set_math

pytestmark = pytest.mark.gpu
RHO_ATOL, DB_ATOL, N_ATOL = 1e-5, 2e-4, 2e-6


def run_both(p, st, steps):
    from lb3d_b200.lib import Lattice
    lat = Lattice(p, precision=1)
    lat.upload_state(st)
    lat.time_loop(steps)
    o = Oracle(p, st)
    o.run(steps)
    return lat, lat.download(), o.get(), o


def check(a, b, nc, what):
    err = np.abs(a["rho"] - b["rho"])
    assert err.max() <= RHO_ATOL, f"{what}: rho err {err.max():.3e}"
    assert np.abs(a["n"] - b["n"]).max() <= N_ATOL, f"{what}: n err {np.abs(a['n'] - b['n']).max():.3e}"
    if nc == 3:
        e = np.abs(a["db"] - b["db"]).max()
        assert e <= DB_ATOL, f"{what}: db err {e:.3e}"


@pytest.mark.parametrize("case", ["gyroid", "bodyForce", "wettingWall"])
def test_fp32_reference_cases(case):
    p, st = load_case(case)
    lat, a, b, _ = run_both(p, st, 20)
    check(a, b, p.ncomp, case)


def _params(L, nc, **kw):
    base = dict(nx=L[0], ny=L[1], nz=L[2], ncomp=nc, tau_d=1.0, g_br=0.08, g_bs=-0.006,
                g_ss=-0.0045, beta=10.0, d_0=1.0, bdist=2, restore=1)
    base.update(kw)
    return Params(**base).finalize()


@pytest.mark.parametrize("dims", [(7, 5, 6), (33, 9, 40), (64, 17, 21)])
def test_fp32_ternary_uneven_tiles(dims):
    """Partial tiles in x and y, several z chunks, periodic wrap across tiles."""
    p = _params(dims, 3, g_accn=1e-4, g_accn_min=2, g_accn_max=4)
    st = uniform_mixture(*dims, 3, seed=7)
    lat, a, b, _ = run_both(p, st, 12)
    check(a, b, 3, str(dims))


@pytest.mark.parametrize("dims", [(9, 6, 5), (40, 12, 33)])
def test_fp32_binary_rock(dims):
    p = _params(dims, 2, g_wr=-0.1, g_wb=0.05, rock_colour_r=1.0, rock_colour_b=0.5,
                g_accn_x=1e-4)
    st = uniform_mixture(*dims, 2, seed=8)
    rng = np.random.default_rng(3)
    st["rock"] = (rng.random(st["n"].shape[2:]) < 0.2).astype(np.float64)
    lat, a, b, o = run_both(p, st, 15)
    check(a, b, 2, str(dims))
    for field in ("od", "wd", "vel"):
        np.testing.assert_allclose(lat.dump(field), o.dump(field), rtol=0, atol=5e-5, err_msg=field)


def test_fp32_mass_conservation():
    p = _params((32, 24, 20), 3)
    st = uniform_mixture(32, 24, 20, 3, seed=9)
    from lb3d_b200.lib import Lattice
    lat = Lattice(p, precision=1)
    lat.upload_state(st)
    m0, _ = lat.conservation()
    lat.time_loop(200)
    m1, u1 = lat.conservation()
    np.testing.assert_allclose(m1, m0, rtol=2e-6)
    assert np.abs(u1).max() < 1e-3
    assert lat.sanity() == (0, 0)


@pytest.mark.parametrize("nc", [2, 3])
def test_fused_and_split_strategies_agree(nc):
    """The kernel strategies (one fused pass; moments, dipole and collide
    passes; the same with the staged collide pass) evaluate the same per-site
    arithmetic with the same roundings, so they agree bit for bit."""
    from lb3d_b200.lib import Lattice
    dims = (40, 24, 20)
    p = _params(dims, nc, g_accn=1e-4)
    st = uniform_mixture(*dims, nc, seed=12)
    out = []
    for split in (0, 1, 2):
        lat = Lattice(p, precision=1)
        lat.upload_state(st)
        lat.set_launch_shape(32, 8, 16, split)
        assert lat.launch_shape == (32, 8, 16, split)
        lat.time_loop(30)
        out.append(lat.download())
    for o in out[1:]:
        assert np.array_equal(out[0]["n"], o["n"])
        if nc == 3:
            assert np.array_equal(out[0]["db"], o["db"])


@pytest.mark.parametrize("nc,dims,shape,rock", [
    (3, (40, 24, 20), (16, 8, 8), False),
    (3, (7, 5, 6), (16, 8, 4), False),
    (3, (33, 9, 40), (32, 8, 16), False),
    (3, (70, 20, 12), (64, 4, 8), False),
    (2, (40, 12, 33), (16, 16, 8), True),
    (2, (9, 6, 5), (32, 4, 8), True),
])
def test_staged_collide_equals_plain_split(nc, dims, shape, rock):
    """Strategy 2 (asynchronously staged collide pass, own moments summed
    from the staged pulls) must reproduce strategy 1 bit for bit, including
    partial tiles, lattices narrower than a tile, short last z chunks and
    bounce-back."""
    from lb3d_b200.lib import Lattice
    kw = dict(g_accn=1e-4, g_accn_min=2, g_accn_max=4)
    if rock:
        kw.update(g_wr=-0.1, g_wb=0.05, rock_colour_r=1.0, rock_colour_b=0.5)
    p = _params(dims, nc, **kw)
    st = uniform_mixture(*dims, nc, seed=21)
    if rock:
        rng = np.random.default_rng(5)
        st["rock"] = (rng.random(st["n"].shape[2:]) < 0.2).astype(np.float64)
    out = []
    for split in (1, 2):
        lat = Lattice(p, precision=1)
        lat.upload_state(st)
        lat.set_launch_shape(*shape, split)
        assert lat.launch_shape == (*shape, split)
        lat.time_loop(25)
        out.append(lat.download())
    assert np.array_equal(out[0]["n"], out[1]["n"])
    if nc == 3:
        assert np.array_equal(out[0]["db"], out[1]["db"])


def test_fp32_lees_edwards_reference_case():
    """The reference's leesEdwards system through the FP32 path: sheared
    x-halos built in FP64 from the FP32 state each step; the plane offset
    (shear_sum) is host FP64 bookkeeping and equals the oracle's exactly."""
    p, st = load_case("leesEdwards")
    lat, a, b, o = run_both(p, st, 20)
    check(a, b, p.ncomp, "leesEdwards")
    assert lat.lees_edwards[0] == o.shear_sum


@pytest.mark.parametrize("shear_u,omega", [(0.05, 0.0), (-0.3, 0.0), (0.2, 0.31)])
@pytest.mark.parametrize("dims", [(40, 12, 20), (8, 6, 10)])
def test_fp32_lees_edwards_offsets(dims, shear_u, omega):
    """Positive, negative (lelo < 0) and oscillating plane offsets; lattices
    wider than one tile (the halo columns sit in the first and last tile) and
    narrower than one tile."""
    p = _params(dims, 2, boundary_cond=-1, inv_fluid=5, shear_u=shear_u, shear_omega=omega,
                g_accn_x=1e-5)
    st = uniform_mixture(*dims, 2, seed=5)
    st["shear_sum"] = 0.37
    from lb3d_b200.lib import Lattice
    lat = Lattice(p, precision=1)
    lat.upload_state(st)
    o = Oracle(p, st)
    for _ in range(2):
        lat.time_loop(10)
        o.run(10)
        check(lat.download(), o.get(), 2, f"LE {dims} shear_u={shear_u}")
    assert lat.lees_edwards[0] == o.shear_sum


def test_fp32_lees_edwards_limits():
    """The FP32 Lees-Edwards kernels exist for the staged split strategy and
    the moment-field strategy only; the others are refused."""
    from lb3d_b200.lib import Lattice, Lb3dError
    p = _params((16, 8, 8), 2, boundary_cond=-1, inv_fluid=5, shear_u=0.05)
    st = uniform_mixture(16, 8, 8, 2, seed=1)
    lat = Lattice(p, precision=1)
    lat.upload_state(st)
    for split in (0, 1):
        with pytest.raises(Lb3dError):
            lat.set_launch_shape(32, 8, 16, split)


@pytest.mark.parametrize("shear_u,omega", [(0.05, 0.0), (-0.3, 0.0), (0.2, 0.31)])
@pytest.mark.parametrize("split", [2, 3])
def test_fp32_lees_edwards_with_walls(split, shear_u, omega):
    """Binary Lees-Edwards with rock (legal in the reference): rock inside, a
    wall on the first z plane (met through the periodic z wrap, where the
    reference's sheared exchange drops the rock colour) and rock on the
    sheared x planes, whose halo sites are never rock.  Against the FP64
    oracle within the FP32 tolerances, for both strategies that run
    Lees-Edwards lattices."""
    from lb3d_b200.lib import Lattice
    dims = (8, 6, 10)
    p = _params(dims, 2, boundary_cond=-1, inv_fluid=5, shear_u=shear_u, shear_omega=omega,
                g_wr=-0.05, g_wb=0.03, rock_colour_r=0.7, rock_colour_b=0.4)
    st = uniform_mixture(*dims, 2, seed=5)
    rock = np.zeros(dims[::-1])
    rock[0, :, 3:5] = 1.0
    rock[4, 2, 0] = 1.0
    rock[6, 3, 7] = 1.0
    rock[5, 1, 5] = 1.0
    st["rock"] = rock
    st["shear_sum"] = 0.37
    lat = Lattice(p, precision=1)
    lat.upload_state(st)
    lat.set_launch_shape(16, 8, 16, split)
    o = Oracle(p, st)
    for _ in range(2):
        lat.time_loop(10)
        o.run(10)
        check(lat.download(), o.get(), 2, f"LE+rock strategy {split} shear_u={shear_u}")
    assert lat.lees_edwards[0] == o.shear_sum


def test_fp32_lees_edwards_with_walls_strategies_agree():
    from lb3d_b200.lib import Lattice
    dims = (40, 12, 20)
    p = _params(dims, 2, boundary_cond=-1, inv_fluid=5, shear_u=-0.3, g_wr=-0.1, g_wb=0.05,
                rock_colour_r=1.0, rock_colour_b=0.5, g_accn_x=1e-5)
    st = uniform_mixture(*dims, 2, seed=9)
    rng = np.random.default_rng(4)
    st["rock"] = (rng.random(dims[::-1]) < 0.15).astype(np.float64)
    out = []
    for split in (2, 3):
        lat = Lattice(p, precision=1)
        lat.upload_state(st)
        lat.set_launch_shape(32, 4, 16, split)
        lat.time_loop(15)
        out.append(lat.download())
    assert np.array_equal(out[0]["n"], out[1]["n"])


def test_fp32_sanity_velocity_and_sums_on_device():
    """The FP32 path's sanity statistics and conservation sums are reduced on
    the device from the deviations; against the FP64 oracle after 10 steps."""
    p, st = load_case("gyroid")
    lat, a, b, o = run_both(p, st, 10)
    va, vb = lat.sanity_velocity(), o.sanity_velocity()
    np.testing.assert_allclose(va["maxvel"], vb["maxvel"], rtol=0, atol=2e-6)
    np.testing.assert_allclose(va["velsum"], vb["velsum"], rtol=0, atol=1e-3)
    assert va["n_fluid"] == vb["n_fluid"]
    m, u = lat.conservation()
    mo, uo = o.sums()
    np.testing.assert_allclose(m, mo, rtol=2e-6)
    assert lat.sanity() == (0, 0)


@pytest.mark.parametrize("inv_fluid,nc,itype,rock", [
    (12, 2, 0, True), (12, 2, 1, False), (12, 3, -1, False), (12, 3, 0, False), (12, 3, 1, False),
    (11, 2, 0, True), (11, 3, 0, False), (7, 2, 0, True), (8, 2, 0, False)])
def test_fp32_inflow_boundaries(inv_fluid, nc, itype, rock):
    """The stage-8 inflow boundaries on the FP32 path -- Zou-He flux
    (inv_fluid 12, every closure), Zou-He density (11) and the binary
    recolouring (7, 8) -- applied to the staged post-stream deviations of the
    z planes, against the FP64 oracle within the path's tolerances; binary
    cases with rock sites on the boundary planes."""
    dims = (20, 12, 10)
    p = _params(dims, nc, boundary_cond=-1, inv_fluid=inv_fluid, inv_type=itype, pr=0.01,
                pb=-0.004, pg=0.002)
    if inv_fluid == 11:
        p = _params(dims, nc, boundary_cond=-1, inv_fluid=11, fr=0.75, fb=0.62, pr=0.66, pb=0.71,
                    amass_b=1.3)
    st = uniform_mixture(*dims, nc, seed=31)
    if rock:
        r = np.zeros(dims[::-1])
        r[0, 3, 2:6] = 1.0
        r[-1, 7, 11] = 1.0
        r[5, :, 9] = 1.0
        st["rock"] = r
    lat, a, b, _ = run_both(p, st, 20)
    check(a, b, nc, f"inflow {inv_fluid} nc={nc} itype={itype}")


def test_fp32_inflow_runs_the_staged_split_strategy_only():
    from lb3d_b200.lib import Lattice, Lb3dError
    p = _params((16, 8, 8), 2, boundary_cond=-1, inv_fluid=12, pr=0.01, pb=0.0, pg=0.0)
    lat = Lattice(p, precision=1)
    lat.upload_state(uniform_mixture(16, 8, 8, 2, seed=1))
    for split in (0, 1):
        with pytest.raises(Lb3dError):
            lat.set_launch_shape(16, 8, 8, split)
    lat.set_launch_shape(16, 8, 8, 2)
    lat.autotune()
    assert lat.launch_shape[3] == 2


@pytest.mark.parametrize("nc,dims,shape,rock", [
    (3, (40, 24, 20), (32, 8, 16), False),
    (3, (7, 5, 6), (16, 8, 16), False),
    (3, (4, 4, 3), (16, 8, 16), False),
    (3, (33, 9, 40), (32, 4, 16), False),
    (3, (70, 20, 12), (64, 4, 32), False),
    (3, (36, 40, 24), (16, 16, 64), False),
    (2, (40, 12, 33), (16, 16, 16), True),
    (2, (9, 6, 5), (32, 4, 16), True),
    (2, (2, 3, 4), (16, 8, 16), False),
    (2, (64, 24, 20), (32, 8, 32), False),
])
def test_moment_field_strategy_equals_staged_split(nc, dims, shape, rock):
    """Strategy 3 (moment field written by the moments pass, read back as TMA
    boxes with a halo by the dipole/force/equilibrium pass) evaluates every
    quantity as strategy 2 does, so with full relaxation (tau = 1) both give
    the same bits: partial tiles, lattices narrower than a tile or than the
    box halo, short z chunks, body force in a sub-box and bounce-back walls."""
    from lb3d_b200.lib import Lattice
    kw = dict(g_accn=1e-4, g_accn_min=2, g_accn_max=4, g_accn_x=-2e-5)
    if rock:
        kw.update(g_wr=-0.1, g_wb=0.05, rock_colour_r=1.0, rock_colour_b=0.5)
    p = _params(dims, nc, **kw)
    st = uniform_mixture(*dims, nc, seed=23)
    if rock:
        rng = np.random.default_rng(6)
        st["rock"] = (rng.random(st["n"].shape[2:]) < 0.2).astype(np.float64)
    out = []
    for split in (2, 3):
        lat = Lattice(p, precision=1)
        lat.upload_state(st)
        lat.set_launch_shape(*shape, split)
        assert lat.launch_shape == (*shape, split)
        lat.time_loop(25)
        lat.sync()
        out.append(lat.download())
    assert np.array_equal(out[0]["n"], out[1]["n"])
    if nc == 3:
        assert np.array_equal(out[0]["db"], out[1]["db"])


def test_moment_field_strategy_against_oracle():
    """Strategy 3 on the gyroid reference system, against the FP64 oracle
    within the FP32 tolerances."""
    from lb3d_b200.lib import Lattice
    p, st = load_case("gyroid")
    lat = Lattice(p, precision=1)
    lat.upload_state(st)
    lat.set_launch_shape(16, 8, 16, 3)
    lat.time_loop(20)
    o = Oracle(p, st)
    o.run(20)
    check(lat.download(), o.get(), 3, "gyroid, strategy 3")


def test_moment_field_strategy_limits():
    """Strategy 3 writes the equilibrium, so it exists only for fully relaxing
    lattices (tau = 1) without inflow boundaries, and needs two sites across
    x and y (a site and its periodic image in the padded fields); elsewhere
    it is refused and the autotuner never offers it."""
    from lb3d_b200.lib import Lattice, Lb3dError
    cases = [
        (_params((16, 8, 8), 3, tau_r=0.8), 3),
        (_params((16, 8, 8), 2, tau_b=1.2, boundary_cond=-1, inv_fluid=5, shear_u=0.05), 2),
        (_params((16, 8, 8), 2, boundary_cond=-1, inv_fluid=12, pr=0.01, pb=0.0, pg=0.0), 2),
        (_params((1, 8, 8), 3), 3),
    ]
    for p, nc in cases:
        lat = Lattice(p, precision=1)
        lat.upload_state(uniform_mixture(p.nx, p.ny, p.nz, nc, seed=2))
        with pytest.raises(Lb3dError):
            lat.set_launch_shape(16, 8, 16, 3)
        lat.autotune()
        assert lat.launch_shape[3] != 3


@pytest.mark.parametrize("shear_u,omega", [(0.05, 0.0), (-0.3, 0.0), (0.2, 0.31)])
@pytest.mark.parametrize("dims,shape", [((40, 12, 20), (32, 4, 16)), ((8, 6, 10), (16, 8, 16)),
                                        ((64, 24, 18), (64, 4, 16))])
def test_moment_field_strategy_lees_edwards_equals_staged_split(dims, shape, shear_u, omega):
    """Binary Lees-Edwards lattices on strategy 3 (pulls across the sheared
    x boundary in the moments pass, the stage-8 halo psi columns in the
    collide pass) give strategy 2's bits for positive, negative and
    oscillating plane offsets, and the oracle's within the tolerances."""
    from lb3d_b200.lib import Lattice
    p = _params(dims, 2, boundary_cond=-1, inv_fluid=5, shear_u=shear_u, shear_omega=omega,
                g_accn_x=1e-5)
    st = uniform_mixture(*dims, 2, seed=5)
    st["shear_sum"] = 0.37
    out = []
    for split in (2, 3):
        lat = Lattice(p, precision=1)
        lat.upload_state(st)
        lat.set_launch_shape(*shape, split)
        lat.time_loop(15)
        lat.sync()
        out.append(lat.download())
        shear_sum = lat.lees_edwards[0]
    assert np.array_equal(out[0]["n"], out[1]["n"])
    o = Oracle(p, st)
    o.run(15)
    check(out[1], o.get(), 2, f"LE strategy 3 {dims} shear_u={shear_u}")
    assert shear_sum == o.shear_sum
