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
