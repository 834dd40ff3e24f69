"""Batched solves: many QUBO (PRAQ) and JRP (PRIA) instances of uneven size in
one engine (include/reform.h).  One launch per kernel kind covers every active
instance; one op_steps block of the whole batch is one CUDA-graph replay;
finished instances retire between replays.  Every instance's result is
bitwise its solo result in the same precision.
"""

from __future__ import annotations

import ctypes
import math
from ctypes import c_int, c_int64, c_void_p

import numpy as np

from . import _native
from .praq import Solve as QuboSolve, _View as _QuboView
from .pria import Solve as JrpSolve, _arrays as _jrp_arrays


class Batch:
    def __init__(self, precision: str = "mixed", stream: int | None = None):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self._lib = _native.lib()
        h = c_void_p()
        st = self._lib.reform_batch_create(int(precision == "mixed"),
                                           c_void_p(stream) if stream else None, ctypes.byref(h))
        if st != 0:
            raise RuntimeError(f"reform_batch_create failed with status {st}")
        self._h = h
        self.kinds: dict[int, tuple[str, object]] = {}

    def add_qubo(self, instance, parameters=None) -> int:
        view = _QuboView(instance)
        p = parameters or self._lib.praq_default_parameters()
        id_ = self._lib.reform_batch_add_qubo(self._h, ctypes.byref(view.struct), ctypes.byref(p))
        if id_ < 0:
            raise RuntimeError(f"reform_batch_add_qubo failed with status {id_}")
        self.kinds[id_] = ("qubo", instance)
        return id_

    def add_jrp(self, instance, parameters=None) -> int:
        k, k0, h = _jrp_arrays(instance)
        p = parameters or self._lib.pria_params_auto(-1, 1e-8)
        id_ = self._lib.reform_batch_add_jrp(self._h, instance.items, instance.periods,
                                             _native.dptr(k), k0, _native.dptr(h), ctypes.byref(p))
        if id_ < 0:
            raise RuntimeError(f"reform_batch_add_jrp failed with status {id_}")
        self.kinds[id_] = ("jrp", instance)
        return id_

    def add_jrp_demand(self, spec, parameters=None) -> int:
        """A demand-form JRP (instances.JrpSpec: K, K0, rates h_i, demands
        d_it), the packed holding costs built on the device."""
        k = np.ascontiguousarray(spec.order_costs, np.float64)
        rate = np.ascontiguousarray(spec.holding_rate, np.float64)
        demand = np.ascontiguousarray(spec.demand, np.float64)
        p = parameters or self._lib.pria_params_auto(-1, 1e-8)
        id_ = self._lib.reform_batch_add_jrp_demand(self._h, spec.items, spec.periods, _native.dptr(k),
                                                    float(spec.joint_order_cost), _native.dptr(rate),
                                                    _native.dptr(demand), ctypes.byref(p))
        if id_ < 0:
            raise RuntimeError(f"reform_batch_add_jrp_demand failed with status {id_}")
        self.kinds[id_] = ("jrp", spec)
        return id_

    def start(self) -> None:
        st = self._lib.reform_batch_start(self._h)
        if st != 0:
            raise RuntimeError(f"reform_batch_start failed with status {st}")

    def run(self, max_blocks: int = -1) -> None:
        st = self._lib.reform_batch_run(self._h, int(max_blocks))
        if st != 0:
            raise RuntimeError(f"reform_batch_run failed with status {st}")

    def launch(self) -> None:
        st = self._lib.reform_batch_launch(self._h)
        if st != 0:
            raise RuntimeError(f"reform_batch_launch failed with status {st}")

    def sync(self, max_ids: int = 4096) -> tuple[int, list[int]]:
        """Wait for the oldest enqueued block; returns (instances still
        running, ids that finished with it)."""
        ids = (c_int * max_ids)()
        n = c_int(0)
        active = self._lib.reform_batch_sync(self._h, ids, max_ids, ctypes.byref(n))
        if active < 0:
            raise RuntimeError(f"reform_batch_sync failed with status {active}")
        return active, [ids[i] for i in range(n.value)]

    def inflight(self) -> int:
        return int(self._lib.reform_batch_inflight(self._h))

    def status(self, id_: int):
        done, it = c_int(0), c_int64(0)
        lo, up = np.zeros(1), np.zeros(1)
        self._lib.reform_batch_status(self._h, id_, ctypes.byref(done), ctypes.byref(it),
                                      _native.dptr(lo), _native.dptr(up))
        return bool(done.value), int(it.value), float(lo[0]), float(up[0])

    def result_qubo(self, id_: int, want_x: bool = True) -> QuboSolve:
        inst = self.kinds[id_][1]
        x = np.empty(inst.n) if want_x else None
        r = _native.PraqResult()
        st = self._lib.reform_batch_result_qubo(self._h, id_, _native.dptr(x) if x is not None else None,
                                                ctypes.byref(r))
        if st != 0:
            raise RuntimeError(f"reform_batch_result_qubo failed with status {st}")
        return QuboSolve(int(r.status), r.lower, r.upper, int(r.iterations), x)

    def result_jrp(self, id_: int, want_solution: bool = False) -> JrpSolve:
        inst = self.kinds[id_][1]
        n, t = inst.items, inst.periods
        out = [np.empty((n, t, t)) for _ in range(3)] if want_solution else [None] * 3
        info = _native.PriaResultInfo()
        st = self._lib.reform_batch_result_jrp(self._h, id_,
                                               *[(_native.dptr(a) if a is not None else None) for a in out],
                                               ctypes.byref(info))
        if st != 0:
            raise RuntimeError(f"reform_batch_result_jrp failed with status {st}")
        return JrpSolve(0, int(info.iterations), info.primal_objective, info.dual_objective,
                        info.relative_gap, *out)

    def set_warm_qubo(self, id_: int, x=None, y=None) -> None:
        """Warm start of a QUBO added and not yet started (x [n], dual pairs
        y [m, 2] or [2m], instance units; projected)."""
        if self.kinds[id_][0] != "qubo":
            raise ValueError(f"instance {id_} is not a QUBO")
        warm = [None if a is None else np.ascontiguousarray(a, np.float64).ravel() for a in (x, y)]
        st = self._lib.reform_batch_set_warm_qubo(self._h, id_, *[_native.dptr(a) if a is not None else None
                                                                 for a in warm])
        if st != 0:
            raise RuntimeError(f"reform_batch_set_warm_qubo failed with status {st}")

    def point_qubo(self, id_: int) -> tuple[np.ndarray, np.ndarray]:
        """(x [n], dual pairs [m, 2]) of a started QUBO's last check."""
        inst = self.kinds[id_][1]
        m = int(np.asarray(inst.vals).size)
        x, y = np.empty(inst.n), np.empty(2 * max(m, 1))
        st = self._lib.reform_batch_point_qubo(self._h, id_, _native.dptr(x), _native.dptr(y))
        if st != 0:
            raise RuntimeError(f"reform_batch_point_qubo failed with status {st}")
        return x, y[:2 * m].reshape(-1, 2)

    def remove(self, id_: int) -> None:
        st = self._lib.reform_batch_remove(self._h, id_)
        if st != 0:
            raise RuntimeError(f"reform_batch_remove failed with status {st}")

    def device_bytes(self) -> int:
        return int(self._lib.reform_batch_device_bytes(self._h))

    def set_shapes(self, grid_multiplier: int = 0) -> None:
        s = _native.ReformShapes(0, grid_multiplier)
        st = self._lib.reform_batch_set_shapes(self._h, ctypes.byref(s))
        if st != 0:
            raise RuntimeError(f"reform_batch_set_shapes failed with status {st}")

    def autotune(self) -> dict:
        s = _native.ReformShapes()
        st = self._lib.reform_batch_autotune(self._h, ctypes.byref(s))
        if st != 0:
            raise RuntimeError(f"reform_batch_autotune failed with status {st}")
        return {"grid_multiplier": s.grid_multiplier}

    def restart(self) -> None:
        """Cold-start every held instance again (the layouts stay resident)."""
        st = self._lib.reform_batch_restart(self._h)
        if st != 0:
            raise RuntimeError(f"reform_batch_restart failed with status {st}")

    def launches(self) -> int:
        return int(self._lib.reform_batch_launches(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.reform_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class EscalatingBatch:
    """The mixed-precision batch with per-instance precision escalation.

    Instances run with FP32 iterates (the "mixed" engine).  A QUBO whose
    relative gap has not halved over the last `stall_iterations` iterations
    (an FP32 plateau: on hard instances FP32 iterates stop gaining near a 1e-3
    gap) leaves the FP32 engine at its last check and continues in an FP64
    engine, warm-started from that point (both parts feasible, so the warm
    start projects nothing away).  Its result then comes from the FP64 engine,
    with the iterations of both phases.  JRP instances stay in FP32 (their
    FP32 iterates reach 1e-4 on every size class of the workload).

    The interface is the `Batch` one the serving loop uses; ids are this
    object's own.
    """

    def __init__(self, stream: int | None = None, stall_iterations: int = 384,
                 fp64_parameters=None):
        self.b32 = Batch("mixed", stream)
        self.b64: Batch | None = None
        self._stream = stream
        self.stall_iterations = int(stall_iterations)
        self._qp64 = fp64_parameters
        self.where: dict[int, tuple[Batch, int]] = {}     # id -> (engine, engine id)
        self.kinds: dict[int, tuple[str, object]] = {}
        self._track: dict[int, tuple[float, int]] = {}    # id -> (reference gap, its iteration)
        self._offset: dict[int, int] = {}                 # id -> FP32 iterations before escalation
        self._qparams: dict[int, object] = {}
        self._next = 0
        self.escalated: list[int] = []

    # -- adding ------------------------------------------------------------
    def _register(self, kind, inst, eid) -> int:
        i = self._next
        self._next += 1
        self.where[i] = (self.b32, eid)
        self.kinds[i] = (kind, inst)
        return i

    def add_qubo(self, instance, parameters=None) -> int:
        i = self._register("qubo", instance, self.b32.add_qubo(instance, parameters))
        self._track[i] = (math.inf, 0)
        self._qparams[i] = parameters
        if self._qp64 is None and parameters is not None:
            self._qp64 = _native.PraqParameters.from_buffer_copy(parameters)
            self._qp64.use_float32 = 0
        return i

    def add_jrp(self, instance, parameters=None) -> int:
        return self._register("jrp", instance, self.b32.add_jrp(instance, parameters))

    def add_jrp_demand(self, spec, parameters=None) -> int:
        return self._register("jrp", spec, self.b32.add_jrp_demand(spec, parameters))

    def start(self) -> None:
        self.b32.start()
        if self.b64 is not None:
            self.b64.start()

    # -- the loop ----------------------------------------------------------
    def _engines(self):
        return [b for b in (self.b32, self.b64) if b is not None]

    def launch(self) -> None:
        for b in self._engines():
            b.launch()

    def inflight(self) -> int:
        return max(b.inflight() for b in self._engines())

    def _escalate(self, i: int) -> None:
        _, eid = self.where[i]
        inst = self.kinds[i][1]
        _, it, _, _ = self.b32.status(eid)
        x, y = self.b32.point_qubo(eid)
        self.b32.remove(eid)
        if self.b64 is None:
            self.b64 = Batch("fp64", self._stream)
        qp = self._qp64 or _native.lib().praq_default_parameters()
        e64 = self.b64.add_qubo(inst, qp)
        self.b64.set_warm_qubo(e64, x, y)
        self.b64.start()
        self.where[i] = (self.b64, e64)
        self._offset[i] = it
        self._track.pop(i, None)
        self.escalated.append(i)

    def _check_stalls(self) -> None:
        for i, (ref_gap, ref_it) in list(self._track.items()):
            b, eid = self.where[i]
            done, it, lo, up = b.status(eid)
            if done:
                self._track.pop(i)
                continue
            gap = (up - lo) / (1.0 + abs(up) + abs(lo))
            if not (gap > 0.5 * ref_gap):          # halved (or the first check)
                self._track[i] = (gap, it)
            elif it - ref_it >= self.stall_iterations:
                self._escalate(i)

    def sync(self) -> tuple[int, list[int]]:
        """Wait for the oldest block of every engine; returns (instances still
        running, ids that finished)."""
        back = {(id(b), eid): i for i, (b, eid) in self.where.items()}
        finished, active = [], 0
        for b in self._engines():
            if b.inflight():
                a, ids = b.sync()
            else:
                a, ids = sum(1 for (bb, e) in self.where.values() if bb is b and not bb.status(e)[0]), []
            active += a
            finished += [back[(id(b), e)] for e in ids if (id(b), e) in back]
        self._check_stalls()
        return active, finished

    def run(self) -> None:
        """Every instance to termination (escalating as it goes)."""
        while True:
            while self.inflight() < 2:
                self.launch()
            active, _ = self.sync()
            if active == 0 and all(b.status(e)[0] for b, e in self.where.values()):
                break
        for b in self._engines():
            while b.inflight():
                b.sync()

    # -- results -----------------------------------------------------------
    def status(self, i: int):
        b, eid = self.where[i]
        done, it, lo, up = b.status(eid)
        return done, it + self._offset.get(i, 0), lo, up

    def result_qubo(self, i: int, want_x: bool = True):
        b, eid = self.where[i]
        r = b.result_qubo(eid, want_x)
        off = self._offset.get(i, 0)
        return QuboSolve(r.status, r.lower, r.upper, r.iterations + off, r.x) if off else r

    def result_jrp(self, i: int, want_solution: bool = False):
        b, eid = self.where[i]
        return b.result_jrp(eid, want_solution)

    def remove(self, i: int) -> None:
        b, eid = self.where.pop(i)
        b.remove(eid)
        self.kinds.pop(i, None)
        self._track.pop(i, None)
        self._qparams.pop(i, None)
        self._offset.pop(i, None)

    def restart(self) -> None:
        """Every instance back into the FP32 engine, cold (escalated ones are
        re-added there)."""
        for i in list(self.escalated):
            b, eid = self.where[i]
            b.remove(eid)
            inst = self.kinds[i][1]
            self.where[i] = (self.b32, self.b32.add_qubo(inst, self._qparams[i]))
        self.escalated.clear()
        self._offset.clear()
        self.b32.restart()
        self._track = {i: (math.inf, 0) for i, (k, _) in self.kinds.items() if k == "qubo"}

    def device_bytes(self) -> int:
        return sum(b.device_bytes() for b in self._engines())

    def launches(self) -> int:
        return sum(b.launches() for b in self._engines())

    def close(self) -> None:
        for b in self._engines():
            b.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
