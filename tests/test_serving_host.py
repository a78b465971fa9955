"""Host logic of the simulation server (no GPU): admission by HBM budget and
free slots, arrival order with pass-ahead across networks, slot recycling,
retirement, latency bookkeeping -- driven with fake pools and a fake clock."""

from collections import deque

import pytest
import torch

from btorch_b200.serving import SimRequest, SimulationServer


class FakeEvent:
    def __init__(self, pool, tick):
        self.pool, self.tick = pool, tick

    def query(self):
        return self.pool.completed >= self.tick


class FakePool:
    """Same interface as NetworkPool; a tick completes when the test says so."""

    def __init__(self, slots, chunk, c_in=4, words=1, max_inflight=2):
        self.slots, self.chunk, self.c_in, self.words = slots, chunk, c_in, words
        self.free = list(range(slots))
        self.active = {}
        self.inflight = deque()
        self.max_inflight = max_inflight
        self.ticks = 0
        self.completed = 0
        self.admitted = []

    def request_bytes(self, req):
        return req.steps * (self.c_in * 4 + self.words * 4)

    def admit(self, req, now):
        req.slot, req.t_admit, req.pos = self.free.pop(0), now, 0
        self.active[req.slot] = req
        self.admitted.append(req.rid)

    def busy(self):
        return bool(self.active) or bool(self.inflight)

    def can_tick(self):
        return bool(self.active) and len(self.inflight) < self.max_inflight

    def tick(self):
        finished = []
        for slot, req in list(self.active.items()):
            req.pos += min(self.chunk, req.steps - req.pos)
            if req.pos >= req.steps:
                finished.append(req)
                del self.active[slot]
        self.ticks += 1
        self.inflight.append((FakeEvent(self, self.ticks), finished))

    def retire(self, now):
        done = []
        while self.inflight and self.inflight[0][0].query():
            _, fin = self.inflight.popleft()
            for r in fin:
                r.t_done = now
                self.free.append(r.slot)
                done.append(r)
        return done

    def drain_events(self):
        return 0


def req(net, steps, arrival, rid):
    return SimRequest(network=net, stimulus=torch.zeros(steps, 4), arrival=arrival, rid=rid)


class Clock:
    """Advances 1 ms per call; pools complete one tick per call."""

    def __init__(self, pools):
        self.t, self.pools = 0.0, pools

    def __call__(self):
        self.t += 1e-3
        for p in self.pools:
            p.completed += 1
        return self.t


def test_budget_and_slots_gate_admission_in_arrival_order():
    a, b = FakePool(slots=2, chunk=10), FakePool(slots=1, chunk=10)
    pools = {"a": a, "b": b}
    per = a.request_bytes(req("a", 10, 0, -1))
    server = SimulationServer(pools, hbm_budget_bytes=3 * per)
    rs = [req("a", 10, 0.0, 0), req("a", 10, 0.0, 1), req("a", 10, 0.0, 2), req("b", 10, 0.0, 3),
          req("b", 10, 0.0, 4)]
    server.queue.extend(rs)
    server.try_admit(0.0)
    # a has 2 slots (requests 0, 1); request 2 waits for a slot, request 3 passes
    # it for network b; request 4 waits (b full, and the budget of 3 is used)
    assert a.admitted == [0, 1] and b.admitted == [3]
    assert [r.rid for r in server.queue] == [2, 4]
    assert server.used == 3 * per


def test_budget_blocks_even_with_free_slots():
    a = FakePool(slots=4, chunk=10)
    per = a.request_bytes(req("a", 10, 0, -1))
    server = SimulationServer({"a": a}, hbm_budget_bytes=2 * per)
    server.queue.extend([req("a", 10, 0.0, i) for i in range(3)])
    server.try_admit(0.0)
    assert a.admitted == [0, 1] and len(server.queue) == 1


def test_run_serves_everything_and_recycles_slots():
    a, b = FakePool(slots=2, chunk=16), FakePool(slots=1, chunk=16)
    pools = {"a": a, "b": b}
    rs = [req("a" if i % 3 else "b", 20 + 7 * i, 0.002 * i, i) for i in range(12)]
    per_max = max(pools[r.network].request_bytes(r) for r in rs)
    server = SimulationServer(pools, hbm_budget_bytes=3 * per_max)
    rep = server.run(rs, clock=Clock(list(pools.values())), idle_sleep=0.0, synchronize=False)
    assert sorted(r.rid for r in rep.requests) == list(range(12))
    for r in rep.requests:
        assert r.t_admit >= r.arrival and r.t_done > r.t_admit and r.latency > 0
        assert r.pos == r.steps
    assert server.used == 0 and sorted(a.free) == [0, 1] and b.free == [0]
    s = rep.summary()
    assert s["requests"] == 12 and s["p50_ms"] <= s["p99_ms"]


def test_request_larger_than_budget_is_rejected():
    a = FakePool(slots=1, chunk=8)
    server = SimulationServer({"a": a}, hbm_budget_bytes=10)
    with pytest.raises(ValueError):
        server.run([req("a", 100, 0.0, 0)], clock=Clock([a]), synchronize=False)


def test_malformed_stimulus_is_refused_before_serving():
    a = FakePool(slots=2, chunk=10)
    server = SimulationServer({"a": a}, hbm_budget_bytes=1 << 20)
    for bad in (torch.zeros(10, 5), torch.zeros(10), torch.zeros(0, 4)):
        with pytest.raises(ValueError, match="stimulus must be"):
            server.run([SimRequest(network="a", stimulus=bad, rid=7)], clock=Clock([a]))
    with pytest.raises(KeyError):
        server.run([req("nope", 10, 0.0, 8)], clock=Clock([a]))
    assert a.admitted == []
