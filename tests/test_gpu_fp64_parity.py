"""FP64 drop-in path (LB3DC_FP64) on the GPU against the CPU oracle and the
reference's golden vectors.  The device path is designed to be bit-identical
to the oracle run with the same deterministic exp/tanh, so every comparison
here is exact unless stated."""
import numpy as np
import pytest

from lb3d_b200.config import Params
from lb3d_b200.ic import uniform_mixture
from tests._fixtures import CASES, FIELDS, load_case, load_golden
from tests._oracle import Oracle, set_math

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, scope="module")
def _detmath():
    set_math(1)
    yield
    set_math(0)


def _lattice(p, st):
    from lb3d_b200.lib import Lattice
    lat = Lattice(p, precision=0)
    lat.upload_state(st)
    return lat


def assert_state_equal(lat, o, what=""):
    a, b = lat.download(), o.get()
    nc = lat.params.ncomp
    for k in ("n", "rho", "mom"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what} {k}")
    if nc == 3:
        np.testing.assert_array_equal(a["db"], b["db"], err_msg=f"{what} db")
        np.testing.assert_array_equal(a["da"], b["da"], err_msg=f"{what} da")


def test_detmath_device_matches_host_bitwise():
    from lb3d_b200.lib import detmath_eval
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-30, 30, 300000), -np.abs(rng.normal(0.7, 0.4, 300000)),
                        rng.uniform(-745, 709, 10000)])
    for fn in ("exp", "expm1", "tanh"):
        xx = np.abs(x) if fn == "tanh" else x
        np.testing.assert_array_equal(detmath_eval(fn, xx, device=True), detmath_eval(fn, xx))


@pytest.mark.parametrize("case", sorted(CASES))
def test_goldens_on_device(case):
    """testLB3D.sh: 10 steps from the t=0 checkpoint, FP32 dumps byte-equal."""
    p, st = load_case(case)
    lat = _lattice(p, st)
    lat.time_loop(10)
    for field in FIELDS[case]:
        gold = load_golden(case, field)
        mine = lat.dump(field).astype(np.float32)
        np.testing.assert_array_equal(mine, gold, err_msg=f"{case}/{field}")


@pytest.mark.parametrize("case", sorted(CASES))
def test_state_bit_identical_to_oracle(case):
    p, st = load_case(case)
    lat = _lattice(p, st)
    o = Oracle(p, st)
    for _ in range(3):
        lat.time_loop(5)
        o.run(5)
        assert_state_equal(lat, o, case)
    assert lat.timestep == 15
    if p.lees_edwards:
        assert lat.lees_edwards[0] == o.shear_sum


@pytest.mark.parametrize("case", ["gyroid", "wettingWall"])
def test_stage_calls_match_oracle_stages(case):
    """The stage entry points in the reference's call order, one step."""
    p, st = load_case(case)
    lat = _lattice(p, st)
    o = Oracle(p, st)
    for stage in (6, 7, 8, 9):
        if stage == 6:
            lat.force_apply(6)
            lat.bc_apply(6)
        elif stage == 7:
            lat.advection()
        elif stage == 8:
            lat.bc_apply(8)
            lat.force_apply(8)
        else:
            lat.collision()
        o.stage(stage)
    assert_state_equal(lat, o, case)


def _params(L, nc, **kw):
    base = dict(nx=L[0], ny=L[1], nz=L[2], ncomp=nc, tau_d=1.0, g_br=0.08, g_bs=-0.006,
                g_ss=-0.0045, beta=10.0, d_0=1.0, bdist=2, restore=1)
    base.update(kw)
    return Params(**base).finalize()


def test_binary_64cube_1000_steps_parity():
    """Binary 64^3 periodic, g_br=0.08, 1000 steps; the
    plain path must match to 1e-12 relative per site (here: exactly)."""
    p = _params((64, 64, 64), 2)
    st = uniform_mixture(64, 64, 64, 2, seed=1)
    lat = _lattice(p, st)
    o = Oracle(p, st)
    lat.time_loop(1000)
    o.run(1000)
    a, b = lat.download(), o.get()
    rel = np.abs(a["rho"] - b["rho"]) / np.abs(b["rho"])
    assert rel.max() <= 1e-12
    np.testing.assert_array_equal(a["n"], b["n"])


def test_ternary_odd_sizes_body_force():
    p = _params((7, 5, 6), 3, g_accn=1e-4, g_accn_x=-2e-5, g_accn_y=3e-5, g_accn_min=2,
                g_accn_max=4, g_accn_min_x=3, g_accn_max_x=7, g_accn_min_y=1, g_accn_max_y=2)
    st = uniform_mixture(7, 5, 6, 3, seed=3)
    lat = _lattice(p, st)
    o = Oracle(p, st)
    lat.time_loop(40)
    o.run(40)
    assert_state_equal(lat, o, "ternary 7x5x6")
    for field in ("od", "wd", "sur", "dir", "vel", "arr"):
        np.testing.assert_array_equal(lat.dump(field), o.dump(field), err_msg=field)


def test_binary_rock_walls_odd_sizes():
    p = _params((9, 6, 5), 2, g_wr=-0.1, g_wb=0.05, rock_colour_r=1.0, rock_colour_b=0.5,
                tau_r=0.8, tau_b=1.3, amass_b=1.5, g_accn_x=1e-4)
    st = uniform_mixture(9, 6, 5, 2, seed=4)
    rng = np.random.default_rng(9)
    rock = (rng.random((5, 6, 9)) < 0.2).astype(np.float64)
    rock[:, 0, :] = 1.0  # a wall through the y wrap
    st["rock"] = rock
    lat = _lattice(p, st)
    o = Oracle(p, st)
    lat.time_loop(30)
    o.run(30)
    assert_state_equal(lat, o, "binary rock")
    for field in ("od", "wd", "vel", "arr", "rock"):
        np.testing.assert_array_equal(lat.dump(field), o.dump(field), err_msg=field)


@pytest.mark.parametrize("shear_u,omega", [(0.05, 0.0), (-0.3, 0.0), (0.2, 0.31)])
def test_lees_edwards_offsets(shear_u, omega):
    """Positive, negative (lelo < 0) and oscillating plane offsets, with
    rock inside and a rock wall through the y/z halo."""
    p = _params((8, 6, 10), 2, boundary_cond=-1, inv_fluid=5, shear_u=shear_u,
                shear_omega=omega, g_wr=-0.05, rock_colour_r=0.7)
    st = uniform_mixture(8, 6, 10, 2, seed=5)
    rock = np.zeros((10, 6, 8))
    rock[0, :, 3:5] = 1.0
    st["rock"] = rock
    st["shear_sum"] = 0.37
    lat = _lattice(p, st)
    o = Oracle(p, st)
    for _ in range(4):
        lat.time_loop(10)
        o.run(10)
        assert_state_equal(lat, o, f"LE shear_u={shear_u}")
    assert lat.lees_edwards[0] == o.shear_sum
    for field in ("od", "wd", "vel", "arr"):
        np.testing.assert_array_equal(lat.dump(field), o.dump(field), err_msg=field)


def test_conservation_and_sanity():
    p = _params((16, 12, 10), 3)
    st = uniform_mixture(16, 12, 10, 3, seed=6)
    lat = _lattice(p, st)
    o = Oracle(p, st)
    lat.time_loop(20)
    o.run(20)
    m, u = lat.conservation()
    mo, uo = o.sums()
    np.testing.assert_allclose(m, mo, rtol=1e-13, atol=0)
    np.testing.assert_allclose(u, uo, rtol=0, atol=1e-12)
    assert lat.sanity() == (0, 0)


def test_arena_roundtrip_matches_reference_layout():
    p, st = load_case("gyroid")
    lat = _lattice(p, st)
    lat.time_loop(2)
    w = lat.download_sites()
    assert w.shape == (18, 18, 18, 79)
    a = lat.download()
    # n_r of site (x=3,y=4,z=5) sits at whole_N(4,5,6)%n_r
    np.testing.assert_array_equal(w[6, 5, 4, 0:19], a["n"][0, :, 5, 4, 3])
    np.testing.assert_array_equal(w[6, 5, 4, 19], a["rho"][0, 5, 4, 3])
    np.testing.assert_array_equal(w[6, 5, 4, 75:78], a["db"][:, 5, 4, 3])
    lat2 = _lattice(p, st)
    lat2.upload_sites(w, nt=2)
    lat2.time_loop(3)
    lat.time_loop(3)
    np.testing.assert_array_equal(lat2.download()["n"], lat.download()["n"])


def test_error_paths():
    from lb3d_b200.lib import Lattice, Lb3dError
    p = _params((8, 8, 8), 2)
    lat = Lattice(p)
    with pytest.raises(Lb3dError):
        lat.time_loop(1)  # no state loaded
    with pytest.raises(Lb3dError):
        lat.bc_apply(7)


@pytest.mark.parametrize("case", ["gyroid", "wettingWall", "bodyForce"])
def test_sanity_velocity_matches_oracle(case):
    """lbe_sanity_check's velocity statistics on the device: the maxima and
    their sites equal the reference loop's exactly, the velocity sums to
    FP64 rounding (a tree sum against the reference's running sum)."""
    p, st = load_case(case)
    lat = _lattice(p, st)
    o = Oracle(p, st)
    lat.time_loop(5)
    o.run(5)
    a, b = lat.sanity_velocity(), o.sanity_velocity()
    np.testing.assert_array_equal(a["maxvel"], b["maxvel"])
    np.testing.assert_array_equal(a["maxpos"], b["maxpos"])
    np.testing.assert_allclose(a["velsum"], b["velsum"], rtol=1e-11, atol=1e-12)
    assert (a["n_fluid"], a["n_too_fast"]) == (b["n_fluid"], b["n_too_fast"])


def test_sanity_velocity_ties_and_fast_sites():
    """With only rest populations every velocity is exactly zero: the maxima
    tie everywhere and the reported site is the last one of the reference's
    loop.  Then a few sites are given large momenta and counted as too fast."""
    p = _params((9, 7, 5), 2)
    st = uniform_mixture(9, 7, 5, 2, seed=2)
    st["n"][:, 18] = st["n"].sum(axis=1)  # all mass at rest
    st["n"][:, :18] = 0.0
    lat = _lattice(p, st)
    o = Oracle(p, st)
    a, b = lat.sanity_velocity(), o.sanity_velocity()
    np.testing.assert_array_equal(a["maxpos"], b["maxpos"])
    assert tuple(a["maxpos"][0, 0]) == (9, 7, 5)
    assert a["n_too_fast"] == 0
    st2 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    st2["n"][0, 0, 1, 2, 3] += 0.2   # +x population of red at (x=4, y=3, z=2)
    st2["n"][1, 4, 3, 5, 6] += 0.3   # +z population of blue at (x=7, y=6, z=4)
    lat2 = _lattice(p, st2)
    o2 = Oracle(p, st2)
    a, b = lat2.sanity_velocity(), o2.sanity_velocity()
    np.testing.assert_array_equal(a["maxvel"], b["maxvel"])
    np.testing.assert_array_equal(a["maxpos"], b["maxpos"])
    assert a["n_too_fast"] == b["n_too_fast"] == 2


@pytest.mark.parametrize("nc,itype", [(2, 0), (2, 1), (3, -1), (3, 0), (3, 1)])
def test_zouhe_flux_boundaries(nc, itype):
    """Zou-He flux boundaries on the z planes (inv_fluid 12) for every
    closure, binary with rock sites on the boundary planes and ternary,
    bit-identical to the oracle."""
    dims = (10, 7, 9)
    p = _params(dims, nc, boundary_cond=-1, inv_fluid=12, inv_type=itype, pr=0.01, pb=-0.004,
                pg=0.002)
    st = uniform_mixture(*dims, nc, seed=11)
    if nc == 2:
        rock = np.zeros((9, 7, 10))
        rock[0, 2, 3:6] = 1.0
        rock[8, 5, 1] = 1.0
        rock[4, :, 7] = 1.0
        st["rock"] = rock
    lat = _lattice(p, st)
    o = Oracle(p, st)
    for _ in range(3):
        lat.time_loop(5)
        o.run(5)
        assert_state_equal(lat, o, f"zouHe nc={nc} itype={itype}")


@pytest.mark.parametrize("inv_fluid,dims,with_rock", [(7, (10, 7, 9), True), (8, (10, 7, 9), False),
                                                     (7, (6, 5, 3), False), (8, (6, 5, 2), True)])
def test_recolouring_boundaries(inv_fluid, dims, with_rock):
    """Binary recolouring inflow (inv_fluid 7 and 8) on the z planes, with
    rock sites on the recoloured planes and lattices whose bottom and top
    planes coincide (nz = 3, 2), bit-identical to the oracle."""
    p = _params(dims, 2, boundary_cond=-1, inv_fluid=inv_fluid)
    st = uniform_mixture(*dims, 2, seed=17)
    if with_rock:
        rock = np.zeros(dims[::-1])
        rock[0, 2, 1:4] = 1.0
        rock[-1, 4, 5] = 1.0
        st["rock"] = rock
    lat = _lattice(p, st)
    o = Oracle(p, st)
    for _ in range(3):
        lat.time_loop(4)
        o.run(4)
        assert_state_equal(lat, o, f"recolour {inv_fluid} {dims}")


@pytest.mark.parametrize("nc,with_rock", [(2, True), (3, False)])
def test_zouhe_density_boundaries(nc, with_rock):
    """Zou-He density boundaries on the z planes (inv_fluid 11): red and blue
    densities fr, fb at z = 1 and pr, pb at z = nz, with unequal masses so
    the blue F(13) term's amass_r shows, binary with rock sites on the
    boundary planes and ternary (surfactant untouched), bit-identical to the
    oracle."""
    dims = (9, 8, 7)
    p = _params(dims, nc, boundary_cond=-1, inv_fluid=11, fr=0.75, fb=0.62, pr=0.66, pb=0.71,
                amass_b=1.3)
    st = uniform_mixture(*dims, nc, seed=23)
    if with_rock:
        rock = np.zeros((7, 8, 9))
        rock[0, 1, 2:5] = 1.0
        rock[6, 6, 8] = 1.0
        rock[3, :, 4] = 1.0
        st["rock"] = rock
    lat = _lattice(p, st)
    o = Oracle(p, st)
    for _ in range(3):
        lat.time_loop(4)
        o.run(4)
        assert_state_equal(lat, o, f"zouHe density nc={nc}")


def test_recolouring_limits():
    from lb3d_b200.lib import Lattice, Lb3dError
    with pytest.raises(Lb3dError):
        Lattice(_params((8, 8, 1), 2, boundary_cond=-1, inv_fluid=8), precision=0)


def test_zouhe_limits():
    from lb3d_b200.lib import Lattice, Lb3dError
    with pytest.raises(Lb3dError):
        Lattice(_params((8, 8, 1), 2, boundary_cond=-1, inv_fluid=12), precision=0)
