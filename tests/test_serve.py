"""Serving-loop policy on the CPU: the seeded request stream, FIFO admission
by device-memory footprint, LRU eviction of idle contexts, and continuous
batching, driven through a fake backend whose solves finish after a set
number of polls."""
import math

import numpy as np
import pytest

from nektar_b200.serve import Request, Scheduler, make_workload, summarize


class FakeSlot:
    def __init__(self, ctx, log):
        self.ctx, self.log = ctx, log
        self.bytes = ctx.backend.slot_bytes(ctx.key)
        self.left = 0

    def start(self, req):
        self.req = req
        self.left = 1 + req.P  # polls until done
        self.log.append(("start", req.rid))

    def advance(self):
        self.left -= 1
        return self.left <= 0

    def finish(self):
        self.log.append(("finish", self.req.rid))
        return ({"iterations": 10 * self.req.P, "converged": True, "rel_residual": 1e-11,
                 "device_ms": 1.0}, np.full(3, float(self.req.rid)))


class FakeContext:
    def __init__(self, backend, key):
        self.backend, self.key = backend, key
        self.bytes = backend.context_bytes(key) - backend.slot_bytes(key)
        self.idle, self.slots, self.active = [], [], 0
        self.closed = False

    def new_slot(self):
        s = FakeSlot(self, self.backend.log)
        self.slots.append(s)
        return s

    def total_bytes(self):
        return self.bytes + sum(s.bytes for s in self.slots)

    def close(self):
        self.closed = True
        self.backend.log.append(("evict", self.key))


class FakeBackend:
    def __init__(self):
        self.log = []
        self.created = []

    def context_bytes(self, key):
        n, P = key
        return 1000 * n + 100 * P + self.slot_bytes(key)

    def slot_bytes(self, key):
        return 10 * key[0]

    def create_context(self, key):
        self.created.append(key)
        return FakeContext(self, key)


def _reqs(specs):
    return [Request(i, t, n, P, 1.0, 1e-10, False, i) for i, (t, n, P) in enumerate(specs)]


def test_workload_is_seeded_and_in_range():
    a = make_workload(2000, rate=200.0, seed=5)
    b = make_workload(2000, rate=200.0, seed=5)
    assert [(r.n, r.P, r.lam, r.mixed, r.arrival) for r in a] == \
           [(r.n, r.P, r.lam, r.mixed, r.arrival) for r in b]
    n = np.array([r.n for r in a])
    P = np.array([r.P for r in a])
    assert n.min() >= 10 and n.max() <= 40
    assert P.min() == 3 and P.max() == 8
    assert all(0.1 <= r.lam <= 10.0 for r in a)
    assert all((r.tol, r.mixed) in ((1e-8, True), (1e-10, False)) for r in a)
    frac_mixed = np.mean([r.mixed for r in a])
    assert 0.45 < frac_mixed < 0.55
    rate = len(a) / a[-1].arrival
    assert 180 < rate < 220
    # log-uniform element counts: the median of log(n^3) sits mid-range
    med = np.median(np.log(n.astype(float) ** 3))
    assert abs(med - 0.5 * (math.log(1000) + math.log(64000))) < 0.3


def test_all_served_fifo_and_within_budget():
    be = FakeBackend()
    specs = [(0.0005 * i, 2 + i % 3, 2 + i % 4) for i in range(40)]
    reqs = _reqs(specs)
    budget = 9000
    sch = Scheduler(be, budget, max_active=4, keep_x=True, idle_sleep=0)
    res = sch.run(reqs)
    assert [r.rid for r in res] == [q.rid for q in reqs]
    assert all(r.converged for r in res)
    assert all(np.all(r.x == r.rid) for r in res)
    assert sch.peak <= budget
    starts = [rid for ev, rid in be.log if ev == "start"]
    assert starts == sorted(starts)  # FIFO admission
    adm = [r.admitted for r in res]
    assert adm == sorted(adm)
    assert all(r.finished >= r.admitted >= r.arrival - 1e-9 for r in res)
    # at most max_active solves were ever in flight
    inflight, worst = 0, 0
    for ev, _ in be.log:
        if ev == "start":
            inflight += 1
        elif ev == "finish":
            inflight -= 1
        worst = max(worst, inflight)
    assert worst <= 4
    s = summarize(res, reqs)
    assert s["requests"] == 40 and s["converged"] == 40
    assert s["latency_s"]["p99"] >= s["latency_s"]["p50"] > 0


def test_idle_contexts_are_evicted_lru_to_make_room():
    be = FakeBackend()
    # three meshes that do not fit together: each context 2000 + slot 20
    reqs = _reqs([(0.0, 2, 1), (0.0, 2, 1), (0.001, 3, 1), (0.002, 2, 1)])
    sch = Scheduler(be, 3300, max_active=1, idle_sleep=0)
    sch.run(reqs)
    assert ("evict", (2, 1)) in be.log
    assert be.created.count((2, 1)) == 2  # rebuilt after eviction
    assert sch.peak <= 3300


def test_request_larger_than_budget_is_refused():
    be = FakeBackend()
    sch = Scheduler(be, 500, idle_sleep=0)
    with pytest.raises(MemoryError):
        sch.run(_reqs([(0.0, 4, 2)]))


def test_slots_are_reused_per_context():
    be = FakeBackend()
    reqs = _reqs([(0.0001 * i, 2, 2) for i in range(10)])
    sch = Scheduler(be, 10 ** 6, max_active=2, idle_sleep=0)
    sch.run(reqs)
    ctx = sch.contexts[(2, 2)]
    assert len(ctx.slots) <= 2 and be.created == [(2, 2)]


def test_prewarm_builds_contexts_within_budget():
    be = FakeBackend()
    sch = Scheduler(be, 5000, idle_sleep=0)
    built = sch.prewarm([(2, 1), (2, 2), (3, 1)])
    assert built == [(2, 1), (2, 2)] or built == [(2, 1), (2, 2), (3, 1)]
    assert sch.used <= 5000
    for key in built:
        ctx = sch.contexts.get(key)
        assert ctx is None or (ctx.active == 0 and len(ctx.idle) == 1)
