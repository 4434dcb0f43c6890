"""CPU tests of the serving loop's scheduling (pf3d.serve.Server) with a
stand-in for the device batches: FIFO admission under the device-memory
budget, both precisions stepped in the same quantum, retirement at each
request's own step count, latency accounting, and the error for a request
that cannot fit the budget on its own.  The device side of the same loop is
tested in test_batch_gpu.py."""
import itertools
import types

import pytest

from pf3d import PF_FP32, PF_FP64, PFError, PF_E_NONFINITE
from pf3d.serve import Job, Server


class FakeBatch:
    """Slots with a step counter and a target, stepped quantum by quantum."""

    log = []

    def __init__(self, precision, budget, max_slots):
        self.precision = precision
        self.slots = {}
        self.free = itertools.count()
        self.pending = 0

    def add(self, g, p):
        s = next(self.free)
        self.slots[s] = {"it": 0, "target": None, "seeded": False}
        return s

    def init_seeded(self, slot, sites):
        self.slots[slot]["seeded"] = True

    def set_target(self, slot, n):
        self.slots[slot]["target"] = n

    def state(self, slot):
        return types.SimpleNamespace(it=self.slots[slot]["it"])

    def progress(self):
        return {s: st["it"] for s, st in self.slots.items()}

    def step_async(self, n):
        FakeBatch.log.append(("step", self.precision))
        self.pending = n

    def wait(self):
        FakeBatch.log.append(("wait", self.precision))
        for st in self.slots.values():
            st["it"] = min(st["target"], st["it"] + self.pending)
        self.pending = 0
        return 1.0

    blown = set()   # (precision, slot) whose state the watchdog finds non-finite

    def diagnosticos(self, slot):
        assert self.slots[slot]["seeded"]
        if (self.precision, slot) in FakeBatch.blown:
            raise PFError(PF_E_NONFINITE, "cells hold a non-finite phi or c")
        return (1.0, 1.0, 0.0, 2.0, 3.0)

    def track(self, slot):
        return (0.5, 4.0, 10.0)

    def remove(self, slot):
        del self.slots[slot]

    def close(self):
        pass


def _job(jid, steps, prec, arrival, nx=32):
    return Job(jid=jid, nx=nx, ny=nx, nz=nx, steps=steps, precision=prec, T0=920.0, rate=20.0, n_bumps=2,
               AAA=0.01, seed=jid, arrival=arrival)


class Clock:
    def __init__(self, dt):
        self.t, self.dt = 0.0, dt

    def __call__(self):
        self.t += self.dt
        return self.t


def test_fifo_admission_under_budget_and_retirement():
    FakeBatch.log.clear()
    jobs = [_job(0, 40, PF_FP32, 0.0), _job(1, 8, PF_FP64, 0.0), _job(2, 16, PF_FP32, 0.0),
            _job(3, 24, PF_FP32, 0.0), _job(4, 8, PF_FP64, 0.5)]
    size = {0: 50, 1: 30, 2: 40, 3: 20, 4: 30}
    srv = Server(budget_bytes=100, quantum=8, batch_factory=FakeBatch, bytes_of=lambda j: size[j.jid])
    peak = []
    out = srv.run(jobs, clock=Clock(0.01), on_quantum=lambda s, done, waiting: peak.append(s.used))
    assert out["requests"] == 5
    assert max(peak) <= 100 and srv.used == 0
    assert all(not b.slots for b in srv.batches.values())
    # FIFO: a request is never admitted before one that arrived earlier
    order = sorted(jobs, key=lambda j: (j.arrival, j.jid))
    adm = [j.admitted for j in order]
    assert adm == sorted(adm)
    # job 2 (40 B) waits behind the budget until job 1 (8 steps) retires
    j = {x.jid: x for x in jobs}
    assert j[2].admitted >= j[1].done
    for x in jobs:
        assert x.done >= x.admitted >= x.arrival
        assert x.result == (1.0, 1.0, 0.0, 2.0, 3.0) and x.track == (0.5, 4.0, 10.0)
    # every request did exactly its own steps: total cell updates
    assert out["gcell_updates"] == pytest.approx(sum(x.cells * x.steps for x in jobs) / 1e9)
    assert out["p99_s"] >= out["p50_s"] > 0


def test_both_precisions_step_in_the_same_quantum():
    FakeBatch.log.clear()
    jobs = [_job(0, 8, PF_FP32, 0.0), _job(1, 8, PF_FP64, 0.0)]
    srv = Server(budget_bytes=1000, quantum=8, batch_factory=FakeBatch, bytes_of=lambda j: 10)
    srv.run(jobs, clock=Clock(0.01))
    assert FakeBatch.log[:4] == [("step", PF_FP32), ("step", PF_FP64), ("wait", PF_FP32), ("wait", PF_FP64)]


def test_request_larger_than_the_budget_is_an_error():
    srv = Server(budget_bytes=10, quantum=8, batch_factory=FakeBatch, bytes_of=lambda j: 11)
    with pytest.raises(RuntimeError, match="does not fit"):
        srv.run([_job(0, 8, PF_FP32, 0.0)], clock=Clock(0.01))


def test_admission_wait_and_budget_use_are_reported():
    FakeBatch.log.clear()
    FakeBatch.blown.clear()
    jobs = [_job(0, 40, PF_FP32, 0.0), _job(1, 16, PF_FP32, 0.0), _job(2, 8, PF_FP32, 0.0)]
    srv = Server(budget_bytes=100, quantum=8, batch_factory=FakeBatch, bytes_of=lambda j: 60)
    out = srv.run(jobs, clock=Clock(0.01))
    assert out["requests"] == 3 and out["failed"] == 0
    # one request fits at a time: the others wait for memory
    assert out["max_waiting_for_memory"] == 2
    assert out["peak_budget_used_gb"] == pytest.approx(60 / 1e9)
    assert out["admission_wait_p99_s"] >= out["admission_wait_p50_s"] > 0
    j = {x.jid: x for x in jobs}
    assert j[1].admitted >= j[0].done and j[2].admitted >= j[1].done


def test_a_blown_up_request_retires_as_failed():
    FakeBatch.log.clear()
    FakeBatch.blown.clear()
    jobs = [_job(0, 16, PF_FP32, 0.0), _job(1, 16, PF_FP32, 0.0), _job(2, 16, PF_FP64, 0.0)]
    srv = Server(budget_bytes=1000, quantum=8, batch_factory=FakeBatch, bytes_of=lambda j: 10)
    FakeBatch.blown.add((PF_FP32, 1))   # the second FP32 slot (job 1)
    out = srv.run(jobs, clock=Clock(0.01))
    FakeBatch.blown.clear()
    assert out["requests"] == 3 and out["failed"] == 1
    j = {x.jid: x for x in jobs}
    assert j[1].failed and j[1].result == () and j[1].track == ()
    assert not j[0].failed and j[0].result == (1.0, 1.0, 0.0, 2.0, 3.0)
    assert srv.used == 0 and all(not b.slots for b in srv.batches.values())
