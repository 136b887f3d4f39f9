"""Host logic of the serving loop without a GPU: admission in arrival order within the memory
budget and the slot limit, retirement, the report's latency figures, and the request generator.
A stand-in for the device batch finishes each instance after a set number of steps."""
import time

import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import serve


class FakeBatch:
    """The part of paraclaws_b200.batch.Batch the server uses; an instance of side m needs
    steps_for(m) steps and occupies m * m * 100 bytes."""

    created = []
    step_seconds = 0.0  # wall time a step takes

    def __init__(self, max_instances, precision=ctl.PRECISION_FP64, device=0):
        self.max_instances = max_instances
        self.slots = {}           # slot -> [steps needed, steps done]
        self.events = []          # ("add" | "remove", side, active count after the event)
        self.sides = {}
        FakeBatch.created.append(self)

    @staticmethod
    def steps_for(m):
        return 8 + m // 32

    @staticmethod
    def instance_bytes(control, custom=None, precision=None):
        return control.m_xi * control.m_eta * 100

    def add(self, control, q, custom=None):
        slot = next(k for k in range(self.max_instances) if k not in self.slots)
        self.slots[slot] = [self.steps_for(control.m_xi), 0]
        self.sides[slot] = control.m_xi
        self.events.append(("add", control.m_xi, len(self.slots)))
        return slot

    def step(self, n):
        if self.step_seconds:
            time.sleep(self.step_seconds * n)
        for rec in self.slots.values():
            rec[1] = min(rec[0], rec[1] + n)

    def poll(self):
        done = np.full(self.max_instances, -1, dtype=np.int32)
        for slot, (need, have) in self.slots.items():
            done[slot] = 1 if have >= need else 0
        return done, np.zeros(self.max_instances, dtype=np.int32)

    def stats(self, slot):
        return ctl_stats(self.slots[slot][1])

    def download(self, slot):
        return np.zeros((4, 4, 3))

    def remove(self, slot):
        self.events.append(("remove", self.sides.pop(slot), len(self.slots) - 1))
        del self.slots[slot]

    def close(self):
        pass


class ctl_stats:
    def __init__(self, accepted):
        self.accepted = accepted


@pytest.fixture
def fake(monkeypatch):
    FakeBatch.created.clear()
    monkeypatch.setattr(FakeBatch, "step_seconds", 0.0)
    monkeypatch.setattr(serve, "Batch", FakeBatch)
    return FakeBatch


def _requests(sides, arrivals=None):
    arrivals = arrivals or [0.0] * len(sides)
    return [serve.Request(k, ctl.dam_break_control(m), ctl.CustomSettings(), t)
            for k, (m, t) in enumerate(zip(sides, arrivals))]


def test_admission_in_arrival_order_within_budget(fake):
    """Budget for one 512-grid: requests are admitted strictly in arrival order (the 512-grid at
    the head of the queue is not overtaken by the 128-grids behind it, which would fit beside the
    two 256-grids) and the footprint of the active set never exceeds the budget."""
    sides = [256, 256, 512, 128, 128, 256]
    budget = 512 * 512 * 100
    srv = serve.SolveServer(budget_bytes=budget, max_slots=16, steps_per_tick=4)
    rep = srv.run(_requests(sides), max_wall=60.0)
    srv.close()
    b = FakeBatch.created[-1]
    adds = [side for kind, side, _ in b.events if kind == "add"]
    assert adds == [256, 256, 512, 128, 128, 256]
    used = 0
    for kind, side, _ in b.events:
        used += (1 if kind == "add" else -1) * side * side * 100
        assert used <= budget
    assert len(rep.results) == len(sides)
    assert all(r.status == 0 for r in rep.results)
    assert [r.accepted for r in rep.results] == [FakeBatch.steps_for(m) for m in sides]


def test_request_larger_than_the_budget_is_refused_not_blocking(fake):
    """A request whose footprint exceeds the whole budget is answered at once with PCL_ERR_FULL;
    the requests behind it are served."""
    from paraclaws_b200._lib import PCL_ERR_FULL
    sides = [128, 1024, 128]
    srv = serve.SolveServer(budget_bytes=2 * 128 * 128 * 100, max_slots=8, steps_per_tick=4)
    rep = srv.run(_requests(sides), max_wall=60.0)
    srv.close()
    by_id = {r.rid: r for r in rep.results}
    assert sorted(by_id) == [0, 1, 2]
    assert by_id[1].status == PCL_ERR_FULL and by_id[1].accepted == 0
    assert by_id[0].status == 0 and by_id[2].status == 0
    assert rep.summary()["errors"] == 1


def test_slot_limit_caps_the_active_set(fake):
    sides = [128] * 9
    srv = serve.SolveServer(budget_bytes=1e12, max_slots=3, steps_per_tick=2)
    rep = srv.run(_requests(sides), max_wall=60.0)
    srv.close()
    b = FakeBatch.created[-1]
    assert max(n for kind, _, n in b.events if kind == "add") == 3
    assert rep.peak_active == 3
    assert len(rep.results) == 9


def test_later_arrivals_join_running_requests(fake):
    """Continuous batching: a request that arrives while others run is admitted beside them (the
    active set grows past one) and every request finishes."""
    sides = [1024, 128, 128]  # the first needs 40 steps of 1 ms; the others arrive after 1 and 2 ms
    fake.step_seconds = 0.001
    srv = serve.SolveServer(budget_bytes=1e12, max_slots=8, steps_per_tick=1)
    rep = srv.run(_requests(sides, [0.0, 0.001, 0.002]), max_wall=60.0)
    srv.close()
    b = FakeBatch.created[-1]
    assert max(n for kind, _, n in b.events if kind == "add") >= 2
    assert sorted(r.rid for r in rep.results) == [0, 1, 2]
    for r in rep.results:
        assert r.finished >= r.admitted >= r.arrival
        assert r.latency >= r.queued >= 0.0


def test_report_percentiles_are_nearest_rank():
    results = [serve.Result(k, 0.0, 0.0, float(k + 1), 1, 1, 0) for k in range(100)]
    rep = serve.ServeReport(results, 10.0, 100.0, 0, 1, 100)
    assert rep.percentile(50) == 50.0
    assert rep.percentile(99) == 99.0
    assert rep.percentile(100) == 100.0
    s = rep.summary()
    assert s["requests"] == 100 and s["p50_s"] == 50.0 and s["throughput_cell_updates_per_s"] == 10.0


def test_poisson_requests_are_seeded_and_in_range():
    a = serve.poisson_requests(50, rate=5.0, seed=3)
    b = serve.poisson_requests(50, rate=5.0, seed=3)
    c = serve.poisson_requests(50, rate=5.0, seed=4)
    key = lambda rs: [(r.control.m_xi, r.control.time_final, r.arrival, r.custom.dam_radius) for r in rs]
    assert key(a) == key(b) and key(a) != key(c)
    arr = [r.arrival for r in a]
    assert arr[0] == 0.0 and all(x <= y for x, y in zip(arr, arr[1:]))
    for r in a:
        assert r.control.m_xi == r.control.m_eta and r.control.m_xi % 32 == 0 and 128 <= r.control.m_xi <= 2048
        assert 0.1 <= r.control.time_final <= 1.0
    # mean gap close to 1 / rate for a long stream
    long = serve.poisson_requests(4000, rate=5.0, seed=1)
    gaps = np.diff([r.arrival for r in long])
    assert abs(gaps.mean() - 0.2) < 0.02


def test_wall_limit_answers_unfinished_requests_with_a_timeout(fake, monkeypatch):
    """When max_wall runs out, requests still running or queued get a timeout result (their
    latency so far), so the percentiles and the error count include them; requests that had
    not arrived are counted apart."""
    monkeypatch.setattr(FakeBatch, "step_seconds", 0.002)
    sides = [2048, 2048, 64, 64]
    # budget for one large instance: the second large one and the small ones queue behind it
    srv = serve.SolveServer(budget_bytes=2048 * 2048 * 100 * 1.5, max_slots=8, steps_per_tick=4)
    reqs = _requests(sides) + _requests([64], [30.0])
    reqs[-1].rid = 4
    rep = srv.run(reqs, max_wall=0.05)
    srv.close()
    by = {r.rid: r for r in rep.results}
    assert sorted(by) == [0, 1, 2, 3], "every arrived request has a result"
    assert by[0].status == serve.PCL_ERR_TIMEOUT and by[0].accepted > 0  # was running
    assert by[1].status == serve.PCL_ERR_TIMEOUT and by[1].accepted == 0  # never admitted
    s = rep.summary()
    assert s["timed_out"] == 4 and s["errors"] == 4 and s["not_arrived"] == 1
    assert s["p99_s"] >= 0.05 - 1e-3
    assert FakeBatch.created[-1].slots == {}, "timed-out instances are removed from the batch"
