"""Host-side logic of the serving loop against a fake engine (no GPU):
admission in arrival order by footprint, continuous batching, retirement."""
import numpy as np

from lb3d_b200.ensemble import Server, sweep_requests


class FakeEnsemble:
    """Mimics Ensemble's contract: first-fit site ranges, members run
    `steps` steps, step() stops at the first completion."""

    def __init__(self, capacity):
        self.cap = capacity
        self.members = {}
        self.free = [(0, capacity)]
        self.next = 0
        self.admit_order = []

    def admit(self, p, state=None, steps=0, seed=None, **kw):
        n = p.nx * p.ny * p.nz
        for k, (b, ln) in enumerate(self.free):
            if ln >= n:
                self.free[k] = (b + n, ln - n)
                slot = self.next
                self.next += 1
                self.members[slot] = [b, n, steps]
                self.admit_order.append(seed)
                return slot
        return None

    def step(self, k):
        act = [m for m in self.members.values() if m[2] > 0]
        if not act:
            return 0
        c = min([k] + [m[2] for m in act])
        for m in act:
            m[2] -= c
        return c

    def sync(self):
        pass

    def finished(self):
        return [s for s, m in self.members.items() if m[2] == 0]

    def retire(self, slot, shape=None, download=True):
        b, n, _ = self.members.pop(slot)
        self.free.append((b, n))
        self.free.sort()
        merged = []
        for seg in self.free:
            if merged and merged[-1][0] + merged[-1][1] == seg[0]:
                merged[-1] = (merged[-1][0], merged[-1][1] + seg[1])
            else:
                merged.append(seg)
        self.free = merged
        return {"slot": slot}

    # asynchronous retire: the copy lands after one poll; until then the
    # slot's range stays reserved
    def retire_async(self, slot, shape):
        self.members[slot][2] = -1  # no longer listed as finished
        self.copying = getattr(self, "copying", {})
        self.copying[slot] = 1

    def poll(self, slot):
        if self.copying[slot] > 0:
            self.copying[slot] -= 1
            return False
        return True

    def collect(self, slot):
        del self.copying[slot]
        return self.retire(slot)


def test_sweep_requests_deterministic_and_in_range():
    a = sweep_requests(200, seed=5)
    b = sweep_requests(200, seed=5)
    assert [(r.arrival, r.steps, r.params.nx, r.params.g_br) for r in a] == \
           [(r.arrival, r.steps, r.params.nx, r.params.g_br) for r in b]
    assert all(16 <= r.params.nx <= 96 and 500 <= r.steps <= 5000 for r in a)
    assert all(0.06 <= r.params.g_br <= 0.10 and -0.008 <= r.params.g_bs <= -0.002 for r in a)
    gaps = np.diff([0] + [r.arrival for r in a])
    assert 0.002 < gaps.mean() < 0.008  # mean 1/200 s


def test_server_admits_in_order_and_completes_all():
    reqs = sweep_requests(40, seed=2, rate=1e6, lmin=16, lmax=40, steps=(10, 50))
    fake = FakeEnsemble(capacity=3 * 40 ** 3)
    out = Server(fake, chunk=8, download=False).run(reqs, realtime=False)
    assert out["solves"] == 40
    assert fake.admit_order == [r.seed for r in sorted(reqs, key=lambda r: r.arrival)]
    assert all(r.done >= r.admitted for r in reqs)
    assert fake.free == [(0, 3 * 40 ** 3)]


def test_server_asynchronous_retire_frees_ranges_only_after_landing():
    """With downloads the finished members are retired asynchronously; their
    ranges are reused only after the copies land, every request completes
    and the whole capacity is free at the end."""
    reqs = sweep_requests(30, seed=4, rate=1e6, lmin=16, lmax=32, steps=(10, 40))
    fake = FakeEnsemble(capacity=2 * 32 ** 3)
    out = Server(fake, chunk=8, download=True).run(reqs, realtime=False)
    assert out["solves"] == 30
    assert all(r.result is not None and r.done >= r.admitted for r in reqs)
    assert fake.free == [(0, 2 * 32 ** 3)]
    assert not getattr(fake, "copying", {})


def test_server_hands_results_to_the_callback_and_keeps_none():
    """A long request stream must not accumulate results in the server: with
    on_result each result goes to the callback as it lands and none stays on
    its request."""
    reqs = sweep_requests(25, seed=6, rate=1e6, lmin=16, lmax=32, steps=(10, 40))
    fake = FakeEnsemble(capacity=2 * 32 ** 3)
    got = []
    out = Server(fake, chunk=8, download=True,
                 on_result=lambda r, res: got.append((r.rid, res is not None))).run(reqs, realtime=False)
    assert out["solves"] == 25
    assert sorted(g[0] for g in got) == sorted(r.rid for r in reqs)
    assert all(ok for _, ok in got)
    assert all(getattr(r, "result", None) is None for r in reqs)
