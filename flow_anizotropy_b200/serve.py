"""Serving: continuous batching of permeability-tensor requests on one GPU.

Requests (a structure plus its forcing directions) arrive at any time.  The
server keeps one resident ``Batch`` (lbm_batch_* in include/lbm.h): between
CUDA-graph chunks it admits queued requests in arrival order as long as the
HBM budget allows and the resident work (pore voxels x directions advanced
per step) stays under ``max_work``, so newly arrived structures join the
solves already running on the device, and it retires finished ones.  The work
cap keeps just enough solves resident to fill the GPU: beyond it, more
concurrency only slows every resident solve down (all of them finish late
together) without adding throughput.  Every result is the same as the structure
solved alone (the batch's flux reduction is independent of the batch's
contents), and each request's latency is measured from arrival to the end of
the chunk in which its last direction finished.

    srv = Server(precision="fp32", hbm_budget=150 * 2**30)
    rid = srv.submit(solid, forces, Params3D(...))      # non-blocking
    srv.pump()                                           # admit / run a chunk / retire
    done = srv.results()                                 # {rid: [Result3D, ...]}
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from .solver import Batch, LBMError, Params3D


@dataclass
class Request:
    rid: int
    solid: np.ndarray
    forces: np.ndarray
    params: Params3D
    t_arrive: float
    t_admit: float | None = None
    t_done: float | None = None
    results: list | None = None
    work: int = 0                   # pore voxels x directions
    error: str | None = None        # set when the request was rejected (bad input)


@dataclass
class ServeStats:
    latencies: list = field(default_factory=list)       # seconds, arrival -> done
    queue_waits: list = field(default_factory=list)     # seconds, arrival -> admission
    completed: int = 0
    max_resident: int = 0
    max_resident_bytes: int = 0

    def pct(self, p):
        return float(np.percentile(self.latencies, p)) if self.latencies else float("nan")


class Server:
    """Continuous-batching solver for one precision and one device."""

    def __init__(self, precision="fp32", hbm_budget=150 * 2**30, chunk=256, device=0, clock=time.perf_counter,
                 max_work=2_000_000, batch=None, variant=-1):
        # `batch` replaces the device batch (an object with the Batch methods
        # submit/run/poll/resident_bytes/close), for testing the scheduling;
        # `variant` is the step-kernel variant of the batch (-1: the default)
        self.batch = batch if batch is not None else Batch(precision=precision, hbm_budget=hbm_budget,
                                                           chunk=chunk, device=device, variant=variant)
        self.max_work = max_work
        self.resident_work = 0
        self.precision = precision
        self.clock = clock
        self.queue: collections.deque[Request] = collections.deque()
        self.inflight: dict[int, Request] = {}
        self.finished: dict[int, Request] = {}
        self.stats = ServeStats()
        self._next = 0

    def submit(self, solid, forces, params: Params3D, t_arrive: float | None = None) -> int:
        if params.precision != self.precision:
            params = Params3D(**{**params.__dict__, "precision": self.precision})
        rid = self._next
        self._next += 1
        solid = np.ascontiguousarray(solid, np.uint8)
        forces = np.asarray(forces, np.float64).reshape(-1, 3)
        self.queue.append(Request(rid, solid, forces, params, self.clock() if t_arrive is None else t_arrive,
                                  work=int((solid == 0).sum()) * forces.shape[0]))
        return rid

    def _admit(self):
        while self.queue:
            r = self.queue[0]
            if self.inflight and self.max_work and self.resident_work + r.work > self.max_work:
                break                                     # enough work resident to fill the GPU
            try:
                admitted = self.batch.submit(r.solid, r.forces, r.params, tag=r.rid)
            except LBMError as e:
                # this request's input is bad (e.g. no pore space): report it
                # as finished with an error and go on with the queue
                self.queue.popleft()
                r.error, r.t_done = str(e), self.clock()
                self.finished[r.rid] = r
                continue
            if not admitted:
                if not self.inflight:
                    raise RuntimeError(f"request {r.rid} does not fit the HBM budget even alone")
                break                                     # wait for retirements
            self.queue.popleft()
            r.t_admit = self.clock()
            self.inflight[r.rid] = r
            self.resident_work += r.work

    def pump(self, chunks: int = 1):
        """One scheduling round: admit, advance resident solves, retire."""
        self._admit()
        if self.inflight:
            self.batch.run(chunks)
            now_done = self.batch.poll()
            t = self.clock()
            for tag, runs in now_done:
                r = self.inflight.pop(tag)
                self.resident_work -= r.work
                r.results, r.t_done = runs, t
                self.finished[tag] = r
                self.stats.latencies.append(r.t_done - r.t_arrive)
                self.stats.queue_waits.append(r.t_admit - r.t_arrive)
                self.stats.completed += 1
            self.stats.max_resident = max(self.stats.max_resident, len(self.inflight) + len(now_done))
            self.stats.max_resident_bytes = max(self.stats.max_resident_bytes, self.batch.resident_bytes())

    def idle(self) -> bool:
        return not self.queue and not self.inflight

    def drain(self, chunks: int = 1):
        while not self.idle():
            self.pump(chunks)

    def results(self) -> dict:
        return {rid: r.results for rid, r in self.finished.items()}

    def close(self):
        self.batch.close()


def poisson_arrivals(rate: float, duration: float, seed: int = 0):
    """Arrival times of a Poisson process (rate per second) over [0, duration)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(t)


def replay(server: Server, arrivals, make_request, chunks_per_pump: int = 1, horizon: float | None = None):
    """Feed requests at their arrival times (seconds from now) while pumping the
    server; returns the server's stats once every request is done, or, with
    `horizon`, once that many seconds have passed (requests still queued or
    resident then are left unfinished: an overloaded server never drains).
    make_request(i) -> (solid, forces, params)."""
    t0 = server.clock()
    i = 0
    n = len(arrivals)
    while i < n or not server.idle():
        now = server.clock() - t0
        if horizon is not None and now >= horizon:
            break
        while i < n and arrivals[i] <= now:
            solid, forces, params = make_request(i)
            server.submit(solid, forces, params, t_arrive=t0 + arrivals[i])
            i += 1
        if server.idle():
            # nothing resident: sleep until the next arrival
            if i < n:
                time.sleep(max(0.0, min(0.01, arrivals[i] - now)))
            continue
        server.pump(chunks_per_pump)
    return server.stats
