"""The served form's request loop (distributedpanga_b200.serve.Scheduler) on
the host: FIFO admission, the slot limit, the device-memory budget charged at
each slot's high-water footprint, and latency bookkeeping.  A fake executor
stands in for the device."""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from distributedpanga_b200.serve import Request, Scheduler, summarize


class Recorder:
    """An executor that sleeps `dur[rid]` and records what ran when."""

    def __init__(self, dur, sched):
        self.dur = dur
        self.sched = sched
        self.lock = threading.Lock()
        self.running = {}
        self.max_running = 0
        self.max_held = 0
        self.order = []

    def __call__(self, slot, req):
        with self.lock:
            assert slot not in self.running
            self.running[slot] = req.rid
            self.order.append(req.rid)
            self.max_running = max(self.max_running, len(self.running))
            self.max_held = max(self.max_held, sum(self.sched.held))
        time.sleep(self.dur[req.rid])
        with self.lock:
            del self.running[slot]
        return {"query_bases": req.bases, "gdb_bases": req.bases + 1000}


def reqs(arrivals, sizes):
    return [Request(i, b"", a, s) for i, (a, s) in enumerate(zip(arrivals, sizes))]


def test_fifo_and_slot_limit():
    rs = reqs([0.0] * 6, [10] * 6)
    sch = Scheduler(2, 10 ** 9, lambda r: r.bases)
    rec = Recorder({i: 0.1 for i in range(6)}, sch)
    res = sch.run(rs, rec)
    assert rec.order == list(range(6))
    assert rec.max_running == 2
    assert [r.rid for r in res] == list(range(6))
    assert all(r.admitted >= r.arrival - 1e-9 and r.done >= r.admitted for r in res)


def test_budget_limits_concurrency_by_high_water():
    # each request needs 60 of a 100 budget: never two slots growing to 60
    rs = reqs([0.0] * 4, [60] * 4)
    sch = Scheduler(3, 100, lambda r: r.bases)
    rec = Recorder({i: 0.02 for i in range(4)}, sch)
    sch.run(rs, rec)
    assert rec.max_running == 1
    assert rec.max_held <= 100
    # one slot served them all (a slot that already holds 60 is reused)
    assert sorted(sch.held) == [0, 0, 60]


def test_small_requests_share_the_budget():
    rs = reqs([0.0] * 6, [30] * 6)
    sch = Scheduler(3, 100, lambda r: r.bases)
    rec = Recorder({i: 0.2 for i in range(6)}, sch)
    sch.run(rs, rec)
    assert rec.max_running == 3
    assert rec.max_held <= 100


def test_oversized_request_runs_alone():
    rs = reqs([0.0, 0.0, 0.0], [10, 500, 10])
    sch = Scheduler(2, 100, lambda r: r.bases)
    rec = Recorder({0: 0.05, 1: 0.02, 2: 0.02}, sch)
    res = sch.run(rs, rec)
    assert rec.order == [0, 1, 2]
    r0, r1, r2 = res
    assert r1.admitted >= r0.done - 1e-6      # waited for the request in flight
    assert r2.admitted >= r1.done - 1e-6      # FIFO: nothing overtakes it


def test_arrivals_are_waited_for():
    rs = reqs([0.0, 0.5, 1.0], [1, 1, 1])
    sch = Scheduler(4, 10 ** 9, lambda r: r.bases)
    rec = Recorder({i: 0.01 for i in range(3)}, sch)
    res = sch.run(rs, rec)
    for r in res:
        assert r.admitted >= r.arrival - 1e-6   # not before it arrives
        assert r.latency < 0.45                 # nothing queued behind anything
    assert res[2].done >= 1.0


def test_failure_is_raised_after_in_flight_finish():
    done = []

    def ex(slot, req):
        if req.rid == 1:
            raise RuntimeError("request 1 failed")
        time.sleep(0.05)
        done.append(req.rid)
        return {}

    sch = Scheduler(2, 10 ** 9, lambda r: 1)
    with pytest.raises(RuntimeError, match="request 1 failed"):
        sch.run(reqs([0.0, 0.0, 0.5], [1, 1, 1]), ex)
    assert done == [0]                  # request 0 finished; request 2 was never admitted


def test_pick_slot_prefers_slots_that_need_no_growth():
    sch = Scheduler(3, 100, lambda r: r.bases)
    sch.held = [50, 20, 0]
    assert sch.pick_slot([0, 1, 2], 15, 1) == 1      # smallest slot already holding 15
    assert sch.pick_slot([1, 2], 40, 1) == 1         # 20 -> 40 costs 20, the empty slot 40
    assert sch.pick_slot([2], 40, 1) is None         # 50 + 20 + 40 > 100
    assert sch.pick_slot([2], 40, 0) == 2            # nothing in flight: admitted anyway


def test_summary_percentiles():
    from distributedpanga_b200.serve import Result
    res = [Result(i, 0.0, 0.0, float(i + 1), 0, {"query_bases": 10 ** 6, "gdb_bases": 2 * 10 ** 6})
           for i in range(100)]
    s = summarize(res, 50.0)
    lat = np.arange(1, 101, dtype=float)
    assert s["p50_latency_s"] == pytest.approx(np.percentile(lat, 50))
    assert s["p99_latency_s"] == pytest.approx(np.percentile(lat, 99))
    assert s["query_mbp_per_s"] == pytest.approx(2.0)
    assert s["gdb_mbp_per_s"] == pytest.approx(4.0)
