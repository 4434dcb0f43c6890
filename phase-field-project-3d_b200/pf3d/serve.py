"""Batched and served solidification runs.

`batch_domains(seed=3)` draws the batching configuration: 96 independent
domains, x = y log-uniform in [32, 192], z log-uniform in [x, 384], T0 in
[915, 925] K, cooling rate in [5, 40] K/s, 1-16 seed bumps and noise
amplitude in [0, 0.02], all from one seed.

`request_stream(seed=4)` draws the serving configuration: a Poisson stream
(mean 20 requests/s) of requests with x = y log-uniform in [32, 256],
z log-uniform in [x, 512], a step count log-uniform in [500, 20000], FP64
with probability 0.2 and parameters drawn as in the batching configuration.

`Server` is the continuous-batching loop: requests that have arrived are
admitted FIFO while they fit the device-memory budget (their state is
created on the device), every admitted request advances together with the
others in quanta of steps (one pf_batch_step_async per precision, the two
precisions running at the same time on their own streams), and a request
retires -- its diagnostics and its solid fraction and tip position
(evaluated on the device) read back, its memory freed -- as soon as it has
done its steps, which lets the next waiting requests in.  No field ever
leaves the device.  Latency of a request = completion time - arrival time;
its admission wait = admission time - arrival time.  The loop polls the
progress of a whole batch in one library call per quantum.  A request whose
state has gone non-finite (the diagnostics' watchdog, PF_E_NONFINITE) is
retired as failed, without numbers.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import Batch, PF_FP32, PF_FP64, PFError, _abi
from .deck import grid, run6_params
from .init import bump_sites

DX = 0.5e-6


@dataclass
class Job:
    jid: int
    nx: int
    ny: int
    nz: int
    steps: int
    precision: int
    T0: float
    rate: float
    n_bumps: int
    AAA: float
    seed: int
    arrival: float = 0.0
    # filled by the server
    admitted: float = -1.0
    done: float = -1.0
    slot: int = -1
    result: tuple = ()      # diagnostics of the final state (pf_batch_diagnosticos)
    track: tuple = ()       # solid fraction, tip position, solid cells (pf_batch_track)
    failed: bool = False    # the state went non-finite (retired without numbers)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def grid(self):
        return grid(self.nx, self.ny, self.nz, DX)

    def params(self):
        return run6_params(T0=self.T0, taxa_resfr=self.rate, AAA=self.AAA)

    def sites(self):
        return bump_sites(self.nx, self.ny, self.n_bumps, self.seed)


def _loguniform(rng, lo, hi):
    return float(math.exp(rng.uniform(math.log(lo), math.log(hi))))


def _draw_job(rng, jid, xmax, zmax, steps, precision):
    x = int(round(_loguniform(rng, 32, xmax)))
    z = int(round(_loguniform(rng, x, zmax)))
    return Job(jid=jid, nx=x, ny=x, nz=z, steps=steps, precision=precision,
               T0=float(rng.uniform(915.0, 925.0)), rate=float(rng.uniform(5.0, 40.0)),
               n_bumps=int(rng.integers(1, 17)), AAA=float(rng.uniform(0.0, 0.02)), seed=int(rng.integers(1 << 30)))


def batch_domains(seed: int = 3, n: int = 96, steps: int = 3000):
    rng = np.random.default_rng(seed)
    return [_draw_job(rng, j, 192, 384, steps, PF_FP32) for j in range(n)]


def request_stream(seed: int = 4, n: int = 2000, rate_per_s: float = 20.0, step_scale: float = 1.0):
    """The serving configuration; step_scale < 1 shortens every request
    proportionally (a bounded sample of the same stream)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for j in range(n):
        t += float(rng.exponential(1.0 / rate_per_s))
        steps = int(round(_loguniform(rng, 500, 20000)))
        prec = PF_FP64 if rng.uniform() < 0.2 else PF_FP32
        job = _draw_job(rng, j, 256, 512, max(1, int(round(steps * step_scale))), prec)
        job.arrival = t
        jobs.append(job)
    return jobs


def ctx_bytes(job: Job) -> int:
    g = job.grid()
    return int(_abi.LIB.pf_ctx_bytes(C.byref(g), job.precision))


class Server:
    """Continuous batching of solidification requests on one GPU.

    `batch_factory(precision, budget, max_slots)` makes the per-precision
    batches (pf3d.Batch) and `bytes_of(job)` sizes a request's device memory
    (pf_ctx_bytes); both are parameters so that the scheduling can be driven
    by stand-ins on a machine without a GPU."""

    def __init__(self, budget_bytes: float = 150e9, quantum: int = 8, max_slots: int = 4096,
                 batch_factory=Batch, bytes_of=None):
        self.budget = int(budget_bytes)
        self.quantum = quantum
        self.bytes_of = bytes_of if bytes_of is not None else ctx_bytes
        self.batches = {PF_FP32: batch_factory(PF_FP32, 0, max_slots), PF_FP64: batch_factory(PF_FP64, 0, max_slots)}
        self.used = 0
        self.active: dict = {PF_FP32: {}, PF_FP64: {}}   # slot -> job
        self.gcell_updates = 0.0

    def close(self):
        for b in self.batches.values():
            b.close()

    def _admit(self, job: Job, now: float) -> bool:
        need = self.bytes_of(job)
        if self.used + need > self.budget:
            return False
        b = self.batches[job.precision]
        slot = b.add(job.grid(), job.params())
        b.init_seeded(slot, job.sites())
        b.set_target(slot, job.steps)
        job.slot = slot
        job.admitted = now
        self.used += need
        self.active[job.precision][slot] = job
        return True

    def _retire(self, now: float, done: list, progress: dict):
        for prec, b in self.batches.items():
            it = progress.get(prec)
            for slot, job in list(self.active[prec].items()):
                if it is not None and it[slot] >= job.steps:
                    try:
                        job.result = b.diagnosticos(slot)
                        job.track = b.track(slot)
                    except PFError as e:
                        if e.code != _abi.PF_E_NONFINITE:
                            raise
                        job.failed = True
                        job.result = ()
                        job.track = ()
                    job.done = now
                    b.remove(slot)
                    self.used -= self.bytes_of(job)
                    del self.active[prec][slot]
                    done.append(job)

    def run(self, jobs: list, clock=time.perf_counter, on_quantum=None):
        """Serve `jobs` (sorted by arrival, times in seconds from start)."""
        jobs = sorted(jobs, key=lambda j: j.arrival)
        waiting: list = []
        done: list = []
        nxt = 0
        t0 = clock()
        device_ms = 0.0
        peak_used = 0
        waited_for_memory = 0
        while len(done) < len(jobs):
            now = clock() - t0
            while nxt < len(jobs) and jobs[nxt].arrival <= now:
                waiting.append(jobs[nxt])
                nxt += 1
            # FIFO admission while the head fits the budget
            while waiting and self._admit(waiting[0], now):
                waiting.pop(0)
            if waiting:
                waited_for_memory = max(waited_for_memory, len(waiting))
            peak_used = max(peak_used, self.used)
            if not any(self.active.values()):
                if nxt < len(jobs):
                    time.sleep(max(0.0, min(0.01, jobs[nxt].arrival - (clock() - t0))))
                    continue
                if waiting:
                    raise RuntimeError("a request does not fit the device-memory budget on its own")
            # both precisions' quanta run at the same time, each batch on its stream
            stepped = []
            for prec, b in self.batches.items():
                if self.active[prec]:
                    before = b.progress()
                    b.step_async(self.quantum)
                    stepped.append((prec, b, before))
            progress = {}
            for prec, b, before in stepped:
                device_ms += b.wait()
                after = b.progress()
                progress[prec] = after
                self.gcell_updates += sum(job.cells * int(after[s] - before[s])
                                          for s, job in self.active[prec].items()) / 1e9
            self._retire(clock() - t0, done, progress)
            if on_quantum:
                on_quantum(self, done, waiting)
        wall = clock() - t0
        lat = np.array([j.done - j.arrival for j in done])
        adm = np.array([j.admitted - j.arrival for j in done])
        return {"requests": len(done), "failed": sum(1 for j in done if j.failed), "wall_s": wall,
                "device_ms": device_ms, "gcell_updates": self.gcell_updates,
                "gcell_per_s": self.gcell_updates / wall,
                "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "mean_s": float(lat.mean()),
                "admission_wait_p50_s": float(np.percentile(adm, 50)),
                "admission_wait_p99_s": float(np.percentile(adm, 99)),
                "peak_budget_used_gb": peak_used / 1e9, "budget_gb": self.budget / 1e9,
                "max_waiting_for_memory": waited_for_memory}
