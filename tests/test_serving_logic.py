"""Admission and completion logic of the request loop, on CPU, with a fake
batch standing in for the GPU one (no device work)."""
import types

import numpy as np

from mpcns_mercury_b200 import serving as SV


class FakeBatch:
    """Slots with step counters; each run() advances every active slot."""

    def __init__(self, capacity, precision=0):
        self.capacity = capacity
        self.slots = [None] * capacity
        self.log = []

    def add(self, desc):
        s = self.slots.index(None)
        self.slots[s] = {"remaining": 0, "step": 0}
        self.log.append(("add", s))
        return s

    def add_periodic(self, cells, nghost, constants):
        return self.add(None)

    def upload(self, *a, **k):
        pass

    def sync(self, *a):
        pass

    def prepare(self, *a):
        pass

    def request(self, slot, n):
        self.slots[slot]["remaining"] = n

    def run(self, n):
        for _ in range(n):
            for st in self.slots:
                if st and st["remaining"] > 0:
                    st["remaining"] -= 1
                    st["step"] += 1
        self.log.append(("run", n))

    def poll(self):
        return [types.SimpleNamespace(status=0, remaining=(st["remaining"] if st else 0), step=(st["step"] if st else 0))
                for st in self.slots]

    def poll_async(self):
        self.snap = self.poll()
        self.snaps = getattr(self, "snaps", {})
        t = len(self.snaps) % 2
        self.snaps[t] = self.snap
        return t

    def poll_wait(self, t):
        return self.snaps[t]

    def download(self, *a):
        return np.zeros(1)

    def add_like(self, src, constants=None, copy_static=True):
        return self.add(None)

    def remove(self, slot):
        self.slots[slot] = None
        self.log.append(("remove", slot))

    def close(self):
        pass


class FakeDesc:
    def __init__(self, *a, **k):
        pass

    def close(self):
        pass


def _server(monkeypatch, capacity, budget, per_solve):
    monkeypatch.setattr(SV.capi, "Batch", FakeBatch)
    monkeypatch.setattr(SV.capi, "SolveDesc", FakeDesc)
    monkeypatch.setattr(SV, "upload_request", lambda *a, **k: 0)
    monkeypatch.setattr(SV.Server, "_bytes", staticmethod(lambda req, prec, topology=None: per_solve))
    return SV.Server(capacity=capacity, precision=0, hbm_budget=budget, chunk_steps=4)


def _reqs(steps):
    from mpcns_mercury_b200.workloads import STATE_FIELDS

    fields = {name: types.SimpleNamespace(data=None, lo=(0, 0, 0), hi=(1, 1, 1)) for name in STATE_FIELDS}
    return [SV.Request(rid=q, arrival_s=0.0, cells=(8, 8, 8), steps=s, fields=fields) for q, s in enumerate(steps)]


def test_every_request_completes_with_its_steps(monkeypatch):
    srv = _server(monkeypatch, capacity=2, budget=1e12, per_solve=10)
    reqs = _reqs([5, 3, 9, 1, 4])
    stats = srv.serve(reqs)
    assert stats["requests"] == 5
    assert stats["cell_updates"] == 512 * sum(r.steps for r in reqs)
    assert all(r.done_s >= r.admitted_s for r in reqs)
    # never more than `capacity` requests at once (+ the grid's template solve)
    live = 0
    for ev, _ in srv.batch.log:
        live += {"add": 1, "remove": -1}.get(ev, 0)
        assert live <= 2 + 1


def test_admission_respects_the_memory_budget(monkeypatch):
    srv = _server(monkeypatch, capacity=8, budget=35, per_solve=10)  # the template + two requests
    reqs = _reqs([6, 6, 6, 6])
    srv.serve(reqs)
    live = peak = 0
    for ev, _ in srv.batch.log:
        live += {"add": 1, "remove": -1}.get(ev, 0)
        peak = max(peak, live)
    assert peak == 3


def test_completions_are_seen_one_chunk_late(monkeypatch):
    srv = _server(monkeypatch, capacity=4, budget=1e12, per_solve=1)
    reqs = _reqs([2, 10])
    srv.serve(reqs)
    runs = [n for ev, n in srv.batch.log if ev == "run"]
    assert all(n == 4 for n in runs)  # fixed chunks of graph launches
    # the 10-step request needs 3 chunks; its completion is read after the 4th is enqueued
    assert len(runs) == 4


def test_a_request_that_cannot_fit_raises(monkeypatch):
    import pytest

    srv = _server(monkeypatch, capacity=4, budget=15, per_solve=10)  # template + request = 20 > 15
    with pytest.raises(RuntimeError):
        srv.serve(_reqs([3]))
