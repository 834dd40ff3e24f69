"""A continuous-batching request loop: the Python face of the native request
server (include/reform.h, reform_server_*).

Requests (QUBO roof-dual LPs and JRP LPs) arrive over time.  The server's own
host thread keeps the batched engine busy (FP32 iterates with FP64
reductions by default, a QUBO that stalls in FP32 continuing in FP64 from its
last point):

* a request is ADMITTED as soon as the device-memory budget allows (its
  footprint is estimated from its size before it is laid out), between two
  block replays; admission lays the instance out on the device and
  cold-starts it, after which it runs in the same graph replays as everything
  else;
* the engine keeps two op_steps blocks in flight; after each block the server
  reads every instance's control block (one copy) and marks converged
  requests finished;
* `Server.serve` replays an arrival stream in real time, polls for finished
  requests, reads their results (bounds, iterations; a QUBO's primal) and
  RETIRES them, which returns their device memory to the budget; latency is
  measured from a request's arrival to the moment its result is on the host;
  throughput is completed solves per second of wall clock.

`sequential_fifo` is the comparator: the same requests served one at a time
by the plain single-instance FP64 solver, as a FIFO queue, from each request's
measured end-to-end service time.
"""

from __future__ import annotations

import ctypes
import math
import time
from collections import deque
from ctypes import c_int, c_int64, c_void_p
from dataclasses import dataclass, field

import numpy as np

from . import _native, praq, pria
from .instances import JrpSpec, QuboInstance


@dataclass
class Request:
    rid: int
    arrival: float                # seconds after the start of the run
    instance: object              # QuboInstance, JrpSpec or JrpInstance
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
    escalated: bool = False

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def gap(self) -> float:
        return (self.upper - self.lower) / (1.0 + abs(self.upper) + abs(self.lower))


def footprint(instance, precision: str = "mixed") -> int:
    """Device bytes an instance will hold once laid out (its iterates, layout
    and partial sums), a little above the solver's own count: the estimate the
    server reserves against its budget."""
    r = 4 if precision == "mixed" else 8
    if isinstance(instance, QuboInstance):
        n, m = instance.n, instance.edges
        return int(m * (12 + 7 * r) + n * (8 + 6 * r) + (n * 32 + m) // 64 * 64 + 4096)
    tp = instance.periods + (instance.periods & 1)
    nd = instance.items * tp * (tp + 1) // 2
    return int(nd * 13 * r + instance.items * tp * 16 + 65536)


STATES = ("waiting", "running", "finished", "failed")


@dataclass
class Server:
    budget_bytes: float = 150e9
    precision: str = "mixed"
    tolerance: float = 1e-4
    max_iter: int = 200_000
    blocks_in_flight: int = 2
    admit_every: int = 4          # blocks between admissions while requests run
    stall_iterations: int = 384
    done: list = field(default_factory=list)

    def __post_init__(self):
        if self.precision not in ("mixed", "fp64"):
            raise ValueError(f"precision must be 'mixed' or 'fp64', not {self.precision!r}")
        self._lib = _native.lib()
        o = self._lib.reform_server_default_options()
        o.budget_bytes = int(self.budget_bytes)
        o.tolerance = float(self.tolerance)
        o.max_iter = int(self.max_iter)
        o.use_float32 = int(self.precision == "mixed")
        o.blocks_in_flight = int(self.blocks_in_flight)
        o.admit_every = int(self.admit_every)
        o.stall_iterations = int(self.stall_iterations)
        h = c_void_p()
        st = self._lib.reform_server_create(ctypes.byref(o), ctypes.byref(h))
        if st != 0:
            raise RuntimeError(f"reform_server_create failed with status {st}")
        self._h = h
        self._pending: dict[int, Request] = {}      # server id -> request
        self._ids = (c_int64 * 1024)()

    def submit(self, request: Request) -> int:
        """Queue a request with the server; returns its server id."""
        inst = request.instance
        if request.kind == "qubo":
            view = praq._View(inst)
            sid = self._lib.reform_server_submit_qubo(self._h, ctypes.byref(view.struct))
        elif isinstance(inst, JrpSpec):
            k = np.ascontiguousarray(inst.order_costs, np.float64)
            rate = np.ascontiguousarray(inst.holding_rate, np.float64)
            demand = np.ascontiguousarray(inst.demand, np.float64)
            sid = self._lib.reform_server_submit_jrp_demand(
                self._h, inst.items, inst.periods, _native.dptr(k), float(inst.joint_order_cost),
                _native.dptr(rate), _native.dptr(demand))
        else:
            k = np.ascontiguousarray(inst.order_costs, np.float64)
            hc = np.ascontiguousarray(inst.holding_costs, np.float64)
            sid = self._lib.reform_server_submit_jrp(self._h, inst.items, inst.periods, _native.dptr(k),
                                                     float(inst.joint_order_cost), _native.dptr(hc))
        if sid < 0:
            raise RuntimeError(f"reform_server_submit failed with status {sid}")
        self._pending[int(sid)] = request
        return int(sid)

    def status(self, sid: int) -> dict:
        s = _native.ServerRequest()
        if self._lib.reform_server_status(self._h, sid, ctypes.byref(s)) != 0:
            raise KeyError(sid)
        out = {name: getattr(s, name) for name, _ in s._fields_}
        out["state"] = STATES[s.state]
        return out

    def collect(self, t0: float, wait: float = 0.0) -> int:
        """Results of the requests that finished (read, then retired); waits
        up to `wait` seconds for one.  Returns how many completed."""
        count = c_int(0)
        st = self._lib.reform_server_poll(self._h, self._ids, len(self._ids), ctypes.byref(count),
                                          float(wait))
        if st < 0:
            raise RuntimeError(f"the request server stopped with status {st}")
        for k in range(count.value):
            sid = int(self._ids[k])
            req = self._pending.pop(sid)
            s = _native.ServerRequest()
            self._lib.reform_server_status(self._h, sid, ctypes.byref(s))
            if s.state != 2:
                raise RuntimeError(f"request {req.rid} failed with status {s.error}")
            if req.kind == "qubo":
                x = np.empty(req.instance.n)
                r = _native.PraqResult()
                if self._lib.reform_server_result_qubo(self._h, sid, _native.dptr(x), ctypes.byref(r)):
                    raise RuntimeError(f"reading request {req.rid} failed")
                lower, upper, iters = r.lower, r.upper, int(r.iterations)
            else:
                info = _native.PriaResultInfo()
                if self._lib.reform_server_result_jrp(self._h, sid, None, None, None, ctypes.byref(info)):
                    raise RuntimeError(f"reading request {req.rid} failed")
                lower, upper, iters = info.dual_objective, info.primal_objective, int(info.iterations)
            finished = time.perf_counter() - t0
            self._lib.reform_server_retire(self._h, sid)
            self.done.append(Completion(req.rid, req.kind, req.arrival,
                                        req.arrival + max(0.0, s.admitted - s.arrival), finished, iters,
                                        lower, upper, bool(s.escalated)))
        return count.value

    def serve(self, requests: list[Request], t0: float | None = None) -> list[Completion]:
        """Replay `requests` in real time (arrival offsets from t0) and serve
        them; returns the completions in finishing order."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        t0 = time.perf_counter() if t0 is None else t0
        while pending or self._pending:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                self.submit(pending.popleft())
            wait = 0.05 if not pending else max(0.0, min(0.05, pending[0].arrival - now))
            if self._pending:
                self.collect(t0, wait)
            elif pending:
                time.sleep(wait)
        return self.done

    def stats(self) -> dict:
        c = _native.ServerCounts()
        self._lib.reform_server_stats(self._h, ctypes.byref(c))
        return {name: getattr(c, name) for name, _ in c._fields_}

    @property
    def high_water(self) -> int:
        """Most device bytes reserved at once (the budget's high-water mark)."""
        return int(self.stats()["high_water_bytes"])

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.reform_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


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
