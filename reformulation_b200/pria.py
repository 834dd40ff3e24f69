"""PRIA on B200: the Python face of the native JRP solver.

* `Library` mirrors the reference's in-process ctypes wrapper
  (``jrp/harness/pria_cuda_library.py:82-132``): `parameters(**overrides)`
  (pria_params_auto plus overrides) and `solve(instance, parameters)`.
* `DeviceSolver` keeps an instance resident on the GPU (repeat solves, warm
  starts, profiling).
* `solve(instance, *, tolerances, time_limit, ...)` is the backend entry
  point, the drop-in for ``jrp/harness/backends/pria_cuda.py:83-173``.
"""

from __future__ import annotations

import ctypes
import math
import time
from ctypes import c_void_p
from dataclasses import dataclass

import numpy as np

from . import _native
from .results import JrpResult, Tolerances

#: pria_params fields a caller may override (jrp/harness/pria_cuda_library.py:53-54).
SCHEDULE = ("omega", "beta_sufficient", "beta_artificial", "beta_necessary", "theta_initial",
            "theta_target", "theta_decay", "op_steps")


#: reform_pria_run's status when the wall-clock budget ran out (include/pria.h).
TIME_LIMIT = -1


@dataclass(frozen=True)
class Solve:
    """One solve: status (0 or a CUDA error code), bounds, iterations, solution."""

    status: int
    iterations: int
    primal_objective: float
    dual_objective: float
    relative_gap: float
    x: np.ndarray | None = None
    y: np.ndarray | None = None
    z: np.ndarray | None = None


def _arrays(instance):
    k = np.ascontiguousarray(instance.order_costs, dtype=np.float64)
    h = np.ascontiguousarray(instance.holding_costs, dtype=np.float64)
    return k, float(instance.joint_order_cost), h


class Library:
    def __init__(self):
        self._lib = _native.lib()

    def parameters(self, max_iter: int = -1, tolerance: float = 1e-8, **overrides):
        p = self._lib.pria_params_auto(int(max_iter), float(tolerance))
        names = dict(_native.PriaParams._fields_)
        for name, value in overrides.items():
            if name not in names:
                raise KeyError(f"pria_params has no field {name!r}")
            setattr(p, name, value)
        return p

    def solve(self, instance, parameters, precision: str = "fp64", want_solution: bool = False,
              warm=None) -> Solve:
        n, t = instance.items, instance.periods
        info = _native.PriaResultInfo()
        if precision == "fp64":
            k, k0, h = _arrays(instance)
            out = [np.empty((n, t, t)) for _ in range(3)] if want_solution else [None] * 3
            w = [np.ascontiguousarray(a, np.float64) for a in warm] if warm else [None] * 3
            st = self._lib.pria_solve_f64(n, t, _native.dptr(k), k0, _native.dptr(h),
                                          ctypes.byref(parameters),
                                          *[(_native.dptr(a) if a is not None else None) for a in w],
                                          *[(_native.dptr(a) if a is not None else None) for a in out],
                                          ctypes.byref(info))
        else:
            # the f32 ABI takes float32 arrays: converted straight from the
            # instance's own (no copy when it already holds float32)
            kf = np.ascontiguousarray(instance.order_costs, np.float32)
            hf = np.ascontiguousarray(instance.holding_costs, np.float32)
            k0 = float(instance.joint_order_cost)
            out = [np.empty((n, t, t), np.float32) for _ in range(3)] if want_solution else [None] * 3
            w = [np.ascontiguousarray(a, np.float32) for a in warm] if warm else [None] * 3
            st = self._lib.pria_solve_f32(n, t, _native.fptr(kf), ctypes.c_float(k0),
                                          _native.fptr(hf), ctypes.byref(parameters),
                                          *[(_native.fptr(a) if a is not None else None) for a in w],
                                          *[(_native.fptr(a) if a is not None else None) for a in out],
                                          ctypes.byref(info))
        return Solve(int(st), int(info.iterations), info.primal_objective, info.dual_objective,
                     info.relative_gap, *out)

    def objective(self, instance, x) -> float:
        k, k0, h = _arrays(instance)
        x = np.ascontiguousarray(x, np.float64)
        return float(self._lib.pria_objective_f64(instance.items, instance.periods,
                                                  _native.dptr(k), k0, _native.dptr(h),
                                                  _native.dptr(x)))


class DeviceSolver:
    """A JRP instance laid out on the device once and solved repeatedly."""

    KINDS = ("x", "yz", "x_check", "yz_check", "upper", "lower", "check", "restart", "mega_block")

    def __init__(self, instance, parameters=None, precision: str = "fp64", stream: int | None = None):
        self._lib = _native.lib()
        self.items, self.periods = instance.items, instance.periods
        k, k0, h = _arrays(instance)
        self.parameters = parameters or self._lib.pria_params_auto(-1, 1e-8)
        handle = c_void_p()
        st = self._lib.reform_pria_create(self.items, self.periods, _native.dptr(k), k0,
                                          _native.dptr(h), ctypes.byref(self.parameters),
                                          int(precision == "mixed"),
                                          c_void_p(stream) if stream else None, ctypes.byref(handle))
        if st != 0:
            raise RuntimeError(f"reform_pria_create failed with status {st}")
        self._h = handle

    def set_time_limit(self, seconds: float) -> None:
        """Wall-clock budget of each later run (seconds; < 0: none).  A run that
        exceeds it returns TIME_LIMIT with the bracket of its last check."""
        st = self._lib.reform_pria_set_time_limit(self._h, float(seconds))
        if st != 0:
            raise RuntimeError(f"reform_pria_set_time_limit failed with status {st}")

    def set_trace(self, capacity: int) -> None:
        """Later runs record every convergence check (iteration, gap, error,
        omega, bounds, restart decision) into a device ring of `capacity`
        records; 0 turns it off."""
        st = self._lib.reform_pria_set_trace(self._h, int(capacity))
        if st != 0:
            raise RuntimeError(f"reform_pria_set_trace failed with status {st}")
        self._trace_ring = max(int(capacity), 0)

    def trace(self, capacity: int = 1 << 16):
        """The last run's checks, oldest first (a NumPy record array with the
        fields of reform_trace_record)."""
        return _native.read_trace(self._lib.reform_pria_trace, self._h, getattr(self, "_trace_ring", 0), capacity)

    def set_megakernel(self, mode: int = -1) -> bool:
        """-1: automatic (small instances), 0: the per-kernel graph, 1: the
        persistent kernel wherever the instance allows it.  Returns whether
        later runs take the persistent kernel."""
        active = ctypes.c_int(0)
        st = self._lib.reform_pria_set_megakernel(self._h, int(mode), ctypes.byref(active))
        if st != 0:
            raise RuntimeError(f"reform_pria_set_megakernel failed with status {st}")
        return bool(active.value)

    def set_warm(self, x, y, z) -> None:
        self._warm = [np.ascontiguousarray(a, np.float64) for a in (x, y, z)]
        st = self._lib.reform_pria_set_warm(self._h, *[_native.dptr(a) for a in self._warm])
        if st != 0:
            raise RuntimeError(f"reform_pria_set_warm failed with status {st}")

    def run(self) -> int:
        return int(self._lib.reform_pria_run(self._h))

    def result(self, want_solution: bool = False) -> Solve:
        n, t = self.items, self.periods
        out = [np.empty((n, t, t)) for _ in range(3)] if want_solution else [None] * 3
        info = _native.PriaResultInfo()
        st = self._lib.reform_pria_result(self._h,
                                          *[(_native.dptr(a) if a is not None else None) for a in out],
                                          ctypes.byref(info))
        return Solve(int(st), int(info.iterations), info.primal_objective, info.dual_objective,
                     info.relative_gap, *out)

    def run_profiled(self):
        ms = np.zeros(len(self.KINDS))
        count = np.zeros(len(self.KINDS), dtype=np.int64)
        st = self._lib.reform_pria_run_profiled(self._h, _native.dptr(ms), _native.iptr(count))
        return int(st), {k: (float(ms[i]), int(count[i])) for i, k in enumerate(self.KINDS)}

    def launches(self) -> int:
        return int(self._lib.reform_pria_launches(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.reform_pria_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def solve_arrays(instance, tolerance: float = 1e-4, max_iter: int = -1, precision: str = "fp64"):
    """One solve on a fresh DeviceSolver; a dict of the result's numbers."""
    lib = Library()
    with DeviceSolver(instance, lib.parameters(max_iter, tolerance), precision) as dev:
        st = dev.run()
        r = dev.result()
    return dict(status=st, iterations=r.iterations, upper=r.primal_objective,
                lower=r.dual_objective, gap=r.relative_gap)


def solve(instance, *, tolerances: Tolerances = Tolerances(), time_limit: float = math.inf,
          sample_memory: bool = False, precision: str = "fp64", max_iter: int | None = None,
          **schedule) -> JrpResult:
    """Solve the JRP LP of `instance` on the GPU (the reference backend's
    contract: only `tolerances.optimality` reaches the solver; `objective` is
    the upper bound of an optimal run and NaN otherwise).  `time_limit` is a
    wall-clock budget in seconds for set-up and solve together, checked on the
    host at every convergence check: past it the solve stops and the result is
    status "time_limit" with the bracket of the last check (the reference's
    backend instead kills its solver process, jrp/harness/backends/
    pria_cuda.py:114-145, and records no bounds).  `precision` is "fp64" or
    "mixed" (FP32 iterates, FP64 reductions and bounds)."""
    common = dict(backend="pria-b200", instance=instance.name, family=instance.family,
                  items=instance.items, periods=instance.periods, entries=instance.entries,
                  optimality_tolerance=tolerances.optimality)
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
    unknown = set(schedule) - set(SCHEDULE)
    if unknown:
        raise KeyError(f"not schedule fields: {sorted(unknown)}")
    lib = Library()
    p = lib.parameters(-1 if max_iter is None else int(max_iter), tolerances.optimality, **schedule)
    start = time.perf_counter()
    try:
        dev = DeviceSolver(instance, p, precision)
    except RuntimeError as error:
        return JrpResult(status="error", note=str(error)[:200], **common)
    setup = time.perf_counter() - start
    try:
        if math.isfinite(time_limit):
            dev.set_time_limit(max(0.0, time_limit - setup))
        start = time.perf_counter()
        st = dev.run()
        r = dev.result()
        seconds = time.perf_counter() - start
    finally:
        dev.close()
    timed = dict(iterations=r.iterations, setup_seconds=setup, solve_seconds=seconds, **common)
    if st == TIME_LIMIT:
        return JrpResult(status="time_limit", lower=r.dual_objective, upper=r.primal_objective,
                         note=f"stopped past the {time_limit:g}s limit at relative gap "
                              f"{r.relative_gap:.3g}", **timed)
    if st != 0:
        return JrpResult(status="error", note=f"CUDA status {st}", setup_seconds=setup, **common)
    converged = math.isfinite(r.relative_gap) and r.relative_gap <= tolerances.optimality
    if not converged:
        return JrpResult(status="iteration_limit", lower=r.dual_objective, upper=r.primal_objective,
                         note=f"relative gap {r.relative_gap:.3g}", **timed)
    return JrpResult(status="optimal", objective=r.primal_objective, lower=r.dual_objective,
                     upper=r.primal_objective, note=f"precision {precision}", **timed)
