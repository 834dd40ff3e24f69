"""Batched solves: many QUBO (PRAQ) and JRP (PRIA) instances of uneven size in
one engine (include/reform.h).  One launch per kernel kind covers every active
instance; one op_steps block of the whole batch is one CUDA-graph replay;
finished instances retire between replays.  Every instance's result is
bitwise its solo result in the same precision.
"""

from __future__ import annotations

import ctypes
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

    def remove(self, id_: int) -> None:
        st = self._lib.reform_batch_remove(self._h, id_)
        if st != 0:
            raise RuntimeError(f"reform_batch_remove failed with status {st}")

    def device_bytes(self) -> int:
        return int(self._lib.reform_batch_device_bytes(self._h))

    def set_shapes(self, half_edges_per_lane: int = 0, grid_multiplier: int = 0) -> None:
        s = _native.ReformShapes(half_edges_per_lane, grid_multiplier)
        st = self._lib.reform_batch_set_shapes(self._h, ctypes.byref(s))
        if st != 0:
            raise RuntimeError(f"reform_batch_set_shapes failed with status {st}")

    def autotune(self) -> dict:
        s = _native.ReformShapes()
        st = self._lib.reform_batch_autotune(self._h, ctypes.byref(s))
        if st != 0:
            raise RuntimeError(f"reform_batch_autotune failed with status {st}")
        return {"praq_half_edges_per_lane": s.praq_half_edges_per_lane,
                "grid_multiplier": s.grid_multiplier}

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
