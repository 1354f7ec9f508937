"""Ensemble (many lattices in one persistent kernel) and the serving loop."""
import dataclasses

import numpy as np
import pytest

from lb3d_b200.config import Params
from lb3d_b200.ic import uniform_mixture

pytestmark = pytest.mark.gpu
SHAPE = (16, 8, 16, 2)  # tile 16x8, 16 planes, split strategy with the staged collide


def _p(L, nc=3, **kw):
    base = dict(nx=L[0], ny=L[1], nz=L[2], ncomp=nc, tau_d=1.0, g_br=0.08, g_bs=-0.006,
                g_ss=-0.0045, beta=10.0, d_0=1.0, bdist=2, restore=1, precision=1)
    base.update(kw)
    return Params(**base).finalize()


def test_member_same_alone_and_in_a_mix():
    from lb3d_b200.ensemble import Ensemble
    pa = _p((20, 17, 23), g_br=0.09)
    sta = uniform_mixture(20, 17, 23, 3, seed=5)
    # alone
    e1 = Ensemble(3, capacity_sites=200000, max_lattices=8, shape=SHAPE)
    s = e1.admit(pa, sta, steps=40)
    while e1.stats()["active"]:
        e1.step(1000)
    alone = e1.retire(s, (23, 17, 20))
    # in a mix: others of uneven size admitted before and during the run
    e2 = Ensemble(3, capacity_sites=200000, max_lattices=8, shape=SHAPE)
    others = [((16, 16, 16), 0.07, 60), ((31, 9, 12), 0.1, 15)]
    for k, (dims, g, n) in enumerate(others):
        e2.admit(_p(dims, g_br=g), uniform_mixture(*dims, 3, seed=10 + k), steps=n)
    s2 = e2.admit(pa, sta, steps=40)
    e2.step(7)
    e2.admit(_p((24, 24, 8), g_bs=-0.003), uniform_mixture(24, 24, 8, 3, seed=30), steps=100)
    got = None
    while e2.stats()["active"]:
        e2.step(1000)
        if s2 in e2.finished() and got is None:
            got = e2.retire(s2, (23, 17, 20))
    np.testing.assert_array_equal(got["n"], alone["n"])
    np.testing.assert_array_equal(got["db"], alone["db"])


def test_member_equals_single_lattice_fp32_path():
    from lb3d_b200.ensemble import Ensemble
    from lb3d_b200.lib import Lattice
    p = _p((18, 22, 20))
    st = uniform_mixture(18, 22, 20, 3, seed=8)
    lat = Lattice(p)
    lat.upload_state(st)
    lat.set_launch_shape(*SHAPE)
    lat.time_loop(25)
    ref = lat.download()
    e = Ensemble(3, capacity_sites=100000, max_lattices=4, shape=SHAPE)
    e.admit(_p((7, 7, 7)), uniform_mixture(7, 7, 7, 3, seed=1), steps=25)  # occupies base 0
    s = e.admit(p, st, steps=25)
    while e.stats()["active"]:
        e.step(100)
    got = e.retire(s, (20, 22, 18))
    np.testing.assert_array_equal(got["n"], ref["n"])
    np.testing.assert_array_equal(got["db"], ref["db"])


def test_seeded_admission_matches_host_generator():
    from lb3d_b200.ensemble import Ensemble
    p = _p((12, 10, 9))
    e = Ensemble(3, capacity_sites=5000, max_lattices=2, shape=SHAPE)
    s = e.admit(p, steps=0, seed=77)
    got = e.retire(s, (9, 10, 12))
    ref = uniform_mixture(12, 10, 9, 3, seed=77)
    np.testing.assert_allclose(got["n"], ref["n"], rtol=0, atol=3e-9)
    np.testing.assert_allclose(got["db"], ref["db"], rtol=0, atol=1e-7)


def test_admission_by_footprint_and_first_fit():
    from lb3d_b200.ensemble import Ensemble
    e = Ensemble(3, capacity_sites=3 * 4096, max_lattices=8, shape=SHAPE)
    slots = [e.admit(_p((16, 16, 16)), steps=5, seed=i) for i in range(3)]
    assert None not in slots
    assert e.admit(_p((16, 16, 16)), steps=5, seed=9) is None  # full
    e.retire(slots[1], download=False)
    assert e.admit(_p((8, 16, 16)), steps=5, seed=10) is not None  # fits the hole
    assert e.admit(_p((8, 16, 16)), steps=5, seed=11) is not None
    assert e.stats()["free_sites"] == 0


def test_server_continuous_batching_results_match_alone():
    from lb3d_b200.ensemble import Ensemble, Server, sweep_requests
    reqs = sweep_requests(10, seed=3, rate=2000.0, lmin=12, lmax=24, steps=(20, 60))
    ens = Ensemble(3, capacity_sites=40000, max_lattices=16, shape=SHAPE)
    out = Server(ens, chunk=16).run(reqs)
    assert out["solves"] == 10 and out["p99_s"] >= out["p50_s"] > 0
    # a mid-stream request recomputed alone gives the same populations
    r = reqs[4]
    e1 = Ensemble(3, capacity_sites=40000, max_lattices=2, shape=SHAPE)
    s = e1.admit(r.params, steps=r.steps, seed=r.seed)
    while e1.stats()["active"]:
        e1.step(1000)
    alone = e1.retire(s, (r.params.nz, r.params.ny, r.params.nx))
    np.testing.assert_array_equal(r.result["n"], alone["n"])


def test_async_retire_equals_sync_retire_while_others_step():
    """Two identical members: one retired synchronously, the other
    asynchronously while a third member keeps stepping; the landed results
    are identical and the slot frees only after poll reports the copy."""
    from lb3d_b200.ensemble import Ensemble
    p = _p((20, 18, 16))
    st = uniform_mixture(20, 18, 16, 3, seed=21)
    e = Ensemble(3, capacity_sites=100000, max_lattices=8, shape=SHAPE)
    a = e.admit(p, st, steps=12)
    b = e.admit(p, st, steps=12)
    c = e.admit(_p((24, 20, 18)), uniform_mixture(24, 20, 18, 3, seed=22), steps=60)
    while a not in e.finished():
        e.step(100)
    e.sync()
    got_sync = e.retire(a, (16, 18, 20))
    e.retire_async(b, (16, 18, 20))
    e.step(100)  # the third member keeps going meanwhile
    while not e.poll(b):
        pass
    got_async = e.collect(b)
    np.testing.assert_array_equal(got_async["n"], got_sync["n"])
    np.testing.assert_array_equal(got_async["db"], got_sync["db"])
    assert e.stats()["resident"] == 1
    e.close()


@pytest.mark.parametrize("cap,filler_nz", [(40_000_000, 2300), (80_000_000, 4700)])
def test_member_beyond_2_31_population_offsets_equals_member_at_base_0(cap, filler_nz):
    """Ternary ensembles of 40M and 80M sites of capacity (18 and 36 GB of
    populations): the surfactant populations of a member placed behind a
    128x128xfiller_nz filler lie beyond 2^31 floats (and, at 80M, beyond 2^32)
    from the array start; the larger capacity also runs the moments pass with
    64-bit component offsets.  That member must equal, bit for bit, the same
    member placed at site 0."""
    from lb3d_b200.ensemble import Ensemble
    e = Ensemble(3, capacity_sites=cap, max_lattices=4, shape=(32, 4, 8, 2))
    try:
        small = _p((32, 32, 16))
        a = e.admit(small, seed=7, steps=3)
        filler = e.admit(_p((128, 128, filler_nz)), seed=8, steps=3)
        b = e.admit(small, seed=7, steps=3)
        assert None not in (a, filler, b)
        while e.stats()["active"]:
            e.step(1000)
        ra = e.retire(a, (16, 32, 32))
        rb = e.retire(b, (16, 32, 32))
        np.testing.assert_array_equal(ra["n"], rb["n"])
        np.testing.assert_array_equal(ra["db"], rb["db"])
        assert np.all(np.isfinite(ra["n"]))
    finally:
        e.close()
