"""A continuous-batching request loop over the batched engine.

Requests (QUBO roof-dual LPs and JRP LPs) arrive over time.  The server keeps
one engine (`batch.EscalatingBatch`, FP32 iterates with FP64 reductions by
default, a QUBO that stalls in FP32 continuing in FP64 from its last point):

* a request is ADMITTED as soon as the device-memory budget allows (its
  footprint is estimated from its size before it is laid out), between two
  block replays; admission lays the instance out on the device and cold-starts
  it, after which it runs in the same graph replays as everything else;
* the engine keeps two op_steps blocks in flight; after each block the host
  reads every instance's control block (one copy), and instances that have
  converged RETIRE: their bounds and primal are read back to the host, the
  request completes, its device memory returns to the pool;
* latency is measured from a request's arrival to the moment its result is on
  the host; throughput is completed solves per second of wall clock.

`sequential_fifo` is the comparator: the same requests served one at a time
by the plain single-instance FP64 solver, as a FIFO queue, from each request's
measured end-to-end service time.
"""

from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import praq, pria
from .batch import Batch, EscalatingBatch
from .instances import JrpSpec, QuboInstance


@dataclass
class Request:
    rid: int
    arrival: float                # seconds after the start of the run
    instance: object              # QuboInstance or JrpSpec
    kind: str = ""

    def __post_init__(self):
        if not self.kind:
            self.kind = "qubo" if isinstance(self.instance, QuboInstance) else "jrp"


@dataclass
class Completion:
    rid: int
    kind: str
    arrival: float
    admitted: float
    finished: float
    iterations: int
    lower: float
    upper: float

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def gap(self) -> float:
        return (self.upper - self.lower) / (1.0 + abs(self.upper) + abs(self.lower))


def footprint(instance, precision: str = "mixed") -> int:
    """Device bytes an instance will hold once laid out (its iterates, layout
    and partial sums), a little above the solver's own count."""
    r = 4 if precision == "mixed" else 8
    if isinstance(instance, QuboInstance):
        n, m = instance.n, instance.edges
        return int(m * (12 + 7 * r) + n * (8 + 6 * r) + (n * 32 + m) // 64 * 64 + 4096)
    tp = instance.periods + (instance.periods & 1)
    nd = instance.items * tp * (tp + 1) // 2
    return int(nd * 13 * r + instance.items * tp * 16 + 65536)


@dataclass
class Server:
    budget_bytes: float = 150e9
    precision: str = "mixed"
    tolerance: float = 1e-4
    max_iter: int = 200_000
    blocks_in_flight: int = 2
    admit_every: int = 4          # blocks between admissions while instances run
    batch: Batch | EscalatingBatch = field(init=False)
    waiting: deque = field(default_factory=deque)
    running: dict = field(default_factory=dict)   # engine id -> (Request, admitted time)
    done: list = field(default_factory=list)
    high_water: int = 0

    def __post_init__(self):
        # mixed: FP32 iterates, with QUBOs that stall in FP32 continued in FP64
        self.batch = EscalatingBatch() if self.precision == "mixed" else Batch(self.precision)
        self._qp = praq.Library().parameters(tolerance=self.tolerance, max_iter=self.max_iter,
                                             use_float32=int(self.precision == "mixed"))
        self._jp = pria.Library().parameters(self.max_iter, self.tolerance)
        self._reserved = 0

    def submit(self, request: Request) -> None:
        self.waiting.append(request)

    def _admit(self, now: float) -> bool:
        added = False
        while self.waiting:
            req = self.waiting[0]
            need = footprint(req.instance, self.precision)
            if self.running and self._reserved + need > self.budget_bytes:
                break
            self.waiting.popleft()
            if req.kind == "qubo":
                eid = self.batch.add_qubo(req.instance, self._qp)
            elif isinstance(req.instance, JrpSpec):
                eid = self.batch.add_jrp_demand(req.instance, self._jp)
            else:
                eid = self.batch.add_jrp(req.instance, self._jp)
            self._reserved += need
            self.running[eid] = (req, now, need)
            added = True
        if added:
            self.batch.start()
            self.high_water = max(self.high_water, self.batch.device_bytes())
        return added

    def _finish(self, eid: int, t0: float) -> None:
        req, admitted, need = self.running.pop(eid)
        if req.kind == "qubo":
            r = self.batch.result_qubo(eid, want_x=True)
            lower, upper, iters = r.lower, r.upper, r.iterations
        else:
            r = self.batch.result_jrp(eid)
            lower, upper, iters = r.dual_objective, r.primal_objective, r.iterations
        finished = time.perf_counter() - t0
        self.batch.remove(eid)
        self._reserved -= need
        self.done.append(Completion(req.rid, req.kind, req.arrival, admitted, finished, iters, lower,
                                    upper))

    def serve(self, requests: list[Request], t0: float | None = None) -> list[Completion]:
        """Replay `requests` in real time (arrival offsets from t0) and serve
        them; returns the completions in finishing order."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        t0 = time.perf_counter() if t0 is None else t0
        since_admit = self.admit_every
        while pending or self.waiting or self.running:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                self.submit(pending.popleft())
            # the engine drains before it lays out newcomers, so retire first;
            # while instances run, newcomers are admitted every `admit_every`
            # blocks (each admission empties the pipeline once)
            if self.waiting and (not self.running or since_admit >= self.admit_every):
                since_admit = 0
                while self.batch.inflight():
                    _, ids = self.batch.sync()
                    for eid in ids:
                        self._finish(eid, t0)
                self._admit(now)
            if not self.running:
                if pending:
                    time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - t0)))
                continue
            while self.batch.inflight() < self.blocks_in_flight:
                self.batch.launch()
            _, ids = self.batch.sync()
            since_admit += 1
            for eid in ids:
                self._finish(eid, t0)
            # an instance that terminated at its cold start never enters a block
            for eid in [e for e in self.running if self.batch.status(e)[0]]:
                self._finish(eid, t0)
        while self.batch.inflight():
            self.batch.sync()
        return self.done

    def close(self) -> None:
        self.batch.close()


def service_times_fp64(instances: list, tolerance: float = 1e-4, max_iter: int = 200_000) -> list[float]:
    """End-to-end time of each instance solved alone by the plain FP64 solver
    through its C entry point (host buffers in and out)."""
    out = []
    ql, jl = praq.Library(), pria.Library()
    for inst in instances:
        if isinstance(inst, QuboInstance):
            p = ql.parameters(tolerance=tolerance, max_iter=max_iter)
            t0 = time.perf_counter()
            ql.solve(inst, p)
            out.append(time.perf_counter() - t0)
        else:
            dense = inst.build() if isinstance(inst, JrpSpec) else inst
            p = jl.parameters(max_iter, tolerance)
            t0 = time.perf_counter()
            jl.solve(dense, p)
            out.append(time.perf_counter() - t0)
    return out


def sequential_fifo(arrivals: list[float], service: list[float]) -> list[float]:
    """Latencies of a single server taking requests in arrival order."""
    free, lat = 0.0, []
    for a, s in sorted(zip(arrivals, service)):
        start = max(a, free)
        free = start + s
        lat.append(free - a)
    return lat


def percentiles(values, qs=(50, 99)) -> dict:
    if not len(values):
        return {f"p{q}": math.nan for q in qs}
    return {f"p{q}": float(np.percentile(values, q)) for q in qs}
