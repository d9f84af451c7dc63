"""Host logic of the serving loop (femorax_b200/serving.py) with a fake engine: no GPU.

Checks admission in arrival order under an HBM budget and the engine's own room, continuous
admission while others run, retirement, and the error for a request that cannot fit alone.
"""
import pytest

from femorax_b200 import serving


class FakeResult:
    converged = True


class FakeForce:
    def __init__(self, nbytes):
        self.nbytes = nbytes

    def info(self):
        return {"device_bytes": self.nbytes}


class FakeEngine:
    """Slots that finish after `rounds_needed[id]` rounds; at most `max_slots` at once."""

    def __init__(self, max_slots, rounds_needed):
        self.max_slots = max_slots
        self.rounds_needed = rounds_needed
        self.slots = {}  # slot -> [request id, rounds run]
        self.admitted = []
        self.concurrent = 0

    def try_admit(self, force, b):
        if len(self.slots) >= self.max_slots:
            return None
        s = next(i for i in range(self.max_slots) if i not in self.slots)
        self.slots[s] = [b, 0]
        self.admitted.append(b)
        return s

    def round(self):
        self.concurrent = max(self.concurrent, len(self.slots))
        for v in self.slots.values():
            v[1] += 1
        return len(self.slots)

    def finished(self, s):
        rid, r = self.slots[s]
        return r >= self.rounds_needed[rid]

    def retire(self, s):
        rid, _ = self.slots.pop(s)
        return rid, FakeResult()


def fake_prepare(sizes):
    def prep(req, device):
        return FakeForce(sizes[req.id]), req.id, 1
    return prep


def reqs(n):
    return [serving.Request(i, 1, 1, 1, arrival=0.0) for i in range(n)]


def test_admits_in_arrival_order_and_overlaps():
    eng = FakeEngine(max_slots=3, rounds_needed={0: 5, 1: 1, 2: 2, 3: 1, 4: 1})
    srv = serving.Server(eng, hbm_budget=100, prepare_fn=fake_prepare({i: 10 for i in range(5)}), prep_threads=1)
    served, _ = srv.run(reqs(5), realtime=False)
    assert eng.admitted == [0, 1, 2, 3, 4]
    assert sorted(s.id for s in served) == [0, 1, 2, 3, 4]
    assert eng.concurrent == 3           # several solves on the device at once
    assert [s.x for s in served] == [s.id for s in served]
    assert srv.resident == 0


def test_budget_limits_resident_footprint():
    eng = FakeEngine(max_slots=8, rounds_needed={i: 2 for i in range(4)})
    srv = serving.Server(eng, hbm_budget=25, prepare_fn=fake_prepare({i: 10 for i in range(4)}), prep_threads=1)
    served, _ = srv.run(reqs(4), realtime=False)
    assert len(served) == 4
    assert eng.concurrent == 2           # 2 x 10 bytes fit the budget of 25, 3 do not


def test_request_too_large_for_an_empty_engine():
    class NoRoom(FakeEngine):
        def try_admit(self, force, b):
            return None

    srv = serving.Server(NoRoom(1, {0: 1}), hbm_budget=100, prepare_fn=fake_prepare({0: 10}), prep_threads=1)
    with pytest.raises(RuntimeError):
        srv.run(reqs(1), realtime=False)


class FakeMesh:
    padded = 64
    num_equations = 300


class FakeLane:
    """A J2 cohort finishes `steps` calls of step() after it starts."""

    def __init__(self, steps):
        self.steps = steps
        self.members = []
        self.cohorts = []
        self.k = 0

    @property
    def idle(self):
        return not self.members

    def start(self, members, prepared):
        assert len(members) == len(prepared)
        self.members = list(members)
        self.cohorts.append([m[0].id for m in members])
        self.k = 0

    def step(self):
        self.k += 1
        if self.k < self.steps:
            return []
        out = [(req, foot, adm, req.id, FakeResult()) for req, foot, adm in self.members]
        self.members = []
        return out


class OverlapEngine(FakeEngine):
    """Counts rounds that ran while a J2 cohort was on the device."""

    def __init__(self, max_slots, rounds_needed, lane):
        super().__init__(max_slots, rounds_needed)
        self.lane = lane
        self.overlap = 0

    def round(self):
        if not self.lane.idle:
            self.overlap += 1
        return super().round()


def mixed_prepare(req, device):
    if isinstance(req, serving.J2Request):
        return FakeMesh(), None, 0, 300
    return FakeForce(10), req.id, 1


def test_j2_cohorts_run_beside_static_solves():
    lane = FakeLane(steps=4)
    eng = OverlapEngine(max_slots=4, rounds_needed={i: 6 for i in range(10)}, lane=lane)
    stream = [serving.Request(0, 1, 1, 1), serving.J2Request(1, 1, 1, 20), serving.J2Request(2, 1, 1, 20),
              serving.Request(3, 1, 1, 1), serving.J2Request(4, 1, 1, 20), serving.J2Request(5, 1, 1, 20)]
    srv = serving.Server(eng, hbm_budget=10 ** 9, prepare_fn=mixed_prepare, prep_threads=1, lane=lane, max_cohort=3)
    served, _ = srv.run(stream, realtime=False)
    assert sorted(s.id for s in served) == [0, 1, 2, 3, 4, 5]
    assert lane.cohorts == [[1, 2, 4], [5]]  # arrival order, at most max_cohort per cohort
    assert eng.admitted == [0, 3]
    assert eng.overlap > 0                   # static rounds ran while a cohort was on the device
    assert srv.resident == 0


def test_j2_cohort_holds_one_load_path():
    lane = FakeLane(steps=2)
    eng = FakeEngine(max_slots=1, rounds_needed={})
    stream = [serving.J2Request(0, 1, 1, 20, cycles=1), serving.J2Request(1, 1, 1, 20, cycles=2),
              serving.J2Request(2, 1, 1, 20, cycles=2)]
    srv = serving.Server(eng, hbm_budget=10 ** 9, prepare_fn=mixed_prepare, prep_threads=1, lane=lane)
    served, _ = srv.run(stream, realtime=False)
    assert lane.cohorts == [[0], [1, 2]]
    assert len(served) == 3 and srv.resident == 0


def test_mixed_stream_share_and_sizes():
    s = serving.mixed_stream(200, rate=100.0, j2_share=0.3, seed=3)
    j2 = [r for r in s if isinstance(r, serving.J2Request)]
    assert 40 <= len(j2) <= 80
    assert all(r.nx in (1, 2, 4, 8, 16, 24) and 20 <= r.nz <= 400 and 50e3 <= r.sigma_y <= 200e3 for r in j2)
    assert [r.id for r in s] == list(range(200))
