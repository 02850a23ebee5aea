"""Host logic of the serving loop (fourphonon_b200.serve.run_stream) on the
CPU, against a fake server with a fake clock: FIFO admission limited by
slots and budget, continuous batching (work of all running solves advances in
every tick), latency accounting and the p50/p99 summary."""
import numpy as np

from fourphonon_b200 import serve


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class FakeSolve:
    def __init__(self, work, size):
        self.work = work
        self.size = size


class FakeServer:
    """Slots and a byte budget; each tick costs 1 ms and gives every running
    solve an equal share of `max_items` work items."""

    def __init__(self, clock, slots=2, budget=10):
        self.clock = clock
        self.slots = [None] * slots
        self.budget = budget
        self.used = 0
        self.tick_log = []

    def admit(self, s, T):
        if self.used + s.size > self.budget:
            return None
        for i, x in enumerate(self.slots):
            if x is None:
                self.slots[i] = [s, 0]
                self.used += s.size
                return i
        return None

    def tick(self, max_items):
        run = [i for i, x in enumerate(self.slots) if x is not None and x[1] < x[0].work]
        self.tick_log.append(tuple(run))
        share = max(1, max_items // max(1, len(run)))
        fin = []
        for i in run:
            self.slots[i][1] = min(self.slots[i][0].work, self.slots[i][1] + share)
            if self.slots[i][1] == self.slots[i][0].work:
                fin.append(i)
        self.clock.t += 1e-3
        return fin

    def collect(self, slot):
        s = self.slots[slot][0]
        self.slots[slot] = None
        self.used -= s.size
        return {"n_processes": s.work}


def test_fifo_admission_and_batching():
    clk = FakeClock()
    srv = FakeServer(clk, slots=2, budget=10)
    reqs = [serve.Request(0.0, FakeSolve(10, 4), 300.0, tag="a"),
            serve.Request(0.0005, FakeSolve(40, 4), 300.0, tag="b"),
            serve.Request(0.0006, FakeSolve(10, 4), 300.0, tag="c"),
            serve.Request(0.5, FakeSolve(5, 9), 300.0, tag="d")]
    done, summary = serve.run_stream(srv, reqs, tick_items=10, clock=clk, sleep=clk.sleep)
    by = {r.tag: r for r in done}
    # a and b run together from b's arrival on; c waits for a slot (FIFO)
    assert by["a"].admitted == 0.0
    assert by["c"].admitted >= by["a"].finished
    assert any(len(t) == 2 for t in srv.tick_log)
    # d arrives late, after an idle gap, and needs most of the budget
    assert by["d"].admitted >= 0.5
    assert all(r.finished > r.arrival for r in done)
    lat = np.array([r.latency for r in done])
    assert abs(summary["p50_ms"] - 1e3 * np.percentile(lat, 50)) < 1e-9
    assert summary["p99_ms"] >= summary["p50_ms"]
    assert summary["processes"] == 65
    assert summary["requests"] == 4


def test_budget_blocks_until_collect():
    clk = FakeClock()
    srv = FakeServer(clk, slots=4, budget=5)
    reqs = [serve.Request(0.0, FakeSolve(20, 4), 300.0, tag=i) for i in range(3)]
    done, _ = serve.run_stream(srv, reqs, tick_items=5, clock=clk, sleep=clk.sleep)
    # only one fits the budget at a time: strictly sequential service
    fin = sorted(r.finished for r in done)
    adm = sorted(r.admitted for r in done)
    assert adm[1] >= fin[0] and adm[2] >= fin[1]
    assert all(len(t) == 1 for t in srv.tick_log)


def test_metrics_stream():
    import io
    import json

    clk = FakeClock()
    srv = FakeServer(clk, slots=2, budget=10)
    reqs = [serve.Request(0.001 * i, FakeSolve(10 + i, 3), 300.0, tag=i) for i in range(4)]
    out = io.StringIO()
    done, summary = serve.run_stream(srv, reqs, tick_items=4, clock=clk, sleep=clk.sleep, metrics=out)
    lines = [json.loads(x) for x in out.getvalue().splitlines()]
    assert [x["event"] for x in lines] == ["request"] * 4 + ["summary"]
    by = {r.tag: r for r in done}
    for x in lines[:-1]:
        r = by[x["tag"]]
        assert x["finished_s"] == r.finished and x["admitted_s"] == r.admitted
        assert abs(x["latency_ms"] - 1e3 * r.latency) < 1e-9
        assert x["processes"] == r.solve.work
    assert [x["finished_s"] for x in lines[:-1]] == sorted(x["finished_s"] for x in lines[:-1])
    assert lines[-1]["p99_ms"] == summary["p99_ms"] and lines[-1]["requests"] == 4
