"""PRAQ on B200: the Python face of the native solver.

* `Library` mirrors the reference's in-process ctypes wrapper
  (``qubo/harness/praq_cuda_library.py:90-139``): `parameters(**overrides)`,
  `check_interval(n, parameters)`, `solve(instance, parameters) -> Solve`.
* `DeviceSolver` keeps an instance resident on the GPU and solves it again and
  again from the cold start (the timing harness and the serving engine use it).
* `solve(instance, *, tolerances, time_limit, ...)` is the backend entry point,
  the drop-in for ``qubo/harness/backends/praq_cuda.py:79-167``.
* `solve_warm_start`, `relaxation_bounds` and `persistent_variables` are the
  reference's post-solve API (``qubo/praq-jax/praq/solver.py:348-362,482-611``).
"""

from __future__ import annotations

import ctypes
import math
import time
from ctypes import c_void_p
from dataclasses import dataclass

import numpy as np

from . import _native
from .results import QuboResult, Tolerances

#: PraqParameters fields a caller may override (the reference's SCHEDULE,
#: qubo/harness/praq_cuda_library.py:50-52).
SCHEDULE = ("omega", "beta_sufficient", "beta_necessary", "beta_artificial",
            "theta_initial", "theta_target", "theta_decay", "op_steps",
            "interval_offset", "interval_scale", "interval_power")

STATUS = {0: "optimal", 1: "iteration_limit", 2: "time_limit"}


@dataclass(frozen=True)
class Solve:
    """What one solve returned (the reference's `Solve` record)."""

    status: int
    lower: float
    upper: float
    iterations: int
    x: np.ndarray

    @property
    def gap(self) -> float:
        return (self.upper - self.lower) / (1.0 + abs(self.upper) + abs(self.lower))


class _View:
    """Keeps the contiguous arrays alive while the C struct points at them."""

    def __init__(self, instance):
        self.diag = np.ascontiguousarray(instance.diag, dtype=np.float64)
        self.rows = np.ascontiguousarray(instance.rows, dtype=np.int64)
        self.cols = np.ascontiguousarray(instance.cols, dtype=np.int64)
        self.vals = np.ascontiguousarray(instance.vals, dtype=np.float64)
        self.struct = _native.PraqInstance(int(instance.n), int(self.vals.size),
                                           _native.dptr(self.diag), _native.iptr(self.rows),
                                           _native.iptr(self.cols), _native.dptr(self.vals))


class Library:
    """The native library, with the reference Library's three methods."""

    def __init__(self):
        self._lib = _native.lib()

    def parameters(self, **overrides) -> _native.PraqParameters:
        p = self._lib.praq_default_parameters()
        names = dict(_native.PraqParameters._fields_)
        for name, value in overrides.items():
            if name not in names:
                raise KeyError(f"PraqParameters has no field {name!r}")
            setattr(p, name, value)
        return p

    def check_interval(self, n: int, parameters: _native.PraqParameters) -> int:
        if parameters.op_steps > 0:
            return max(int(parameters.op_steps), 2)
        return int(self._lib.praq_check_interval(n, ctypes.byref(parameters)))

    def solve(self, instance, parameters: _native.PraqParameters) -> Solve:
        view = _View(instance)
        x = np.empty(int(instance.n), dtype=np.float64)
        result = _native.PraqResult()
        status = self._lib.praq_solve(ctypes.byref(view.struct), ctypes.byref(parameters),
                                      _native.dptr(x), ctypes.byref(result))
        return Solve(int(status), result.lower, result.upper, int(result.iterations), x)


class DeviceSolver:
    """An instance laid out on the device once and solved any number of times.

    `stream` is a raw cudaStream_t (e.g. ``torch.cuda.current_stream().cuda_stream``)
    or None for a private stream."""

    def __init__(self, instance, parameters: _native.PraqParameters | None = None,
                 stream: int | None = None):
        self._lib = _native.lib()
        self.n, self.m = int(instance.n), int(np.asarray(instance.vals).size)
        view = _View(instance)
        self.parameters = parameters or self._lib.praq_default_parameters()
        handle = c_void_p()
        rc = self._lib.reform_praq_create(ctypes.byref(view.struct), ctypes.byref(self.parameters),
                                          c_void_p(stream) if stream else None,
                                          ctypes.byref(handle))
        if rc != 0:
            raise RuntimeError(f"reform_praq_create failed with status {rc}")
        self._h = handle

    def set_time_limit(self, seconds: float) -> None:
        self._lib.reform_praq_set_time_limit(self._h, float(seconds))

    def set_warm(self, x=None, y=None) -> None:
        """Start later runs from (x, y) instead of the centroid: x [n] and the
        dual pairs y [m, 2] (or [2m]) in instance units, edge order of the
        instance; both are projected.  None keeps that part cold."""
        self._warm = [None if a is None else np.ascontiguousarray(a, np.float64).ravel() for a in (x, y)]
        if self._warm[0] is not None and self._warm[0].size != self.n:
            raise ValueError("warm x must have n entries")
        if self._warm[1] is not None and self._warm[1].size != 2 * self.m:
            raise ValueError("warm y must have 2m entries")
        rc = self._lib.reform_praq_set_warm(self._h, *[_native.dptr(a) if a is not None else None
                                                       for a in self._warm])
        if rc != 0:
            raise RuntimeError(f"reform_praq_set_warm failed with status {rc}")

    def run(self) -> int:
        return int(self._lib.reform_praq_run(self._h))

    def result(self, want_x: bool = True, want_dual: bool = False):
        x = np.empty(self.n) if want_x else None
        y = np.empty(2 * max(self.m, 1)) if want_dual else None
        r = _native.PraqResult()
        rc = self._lib.reform_praq_result(self._h, _native.dptr(x) if x is not None else None,
                                          _native.dptr(y) if y is not None else None,
                                          ctypes.byref(r))
        if rc != 0:
            raise RuntimeError(f"reform_praq_result failed with status {rc}")
        out = Solve(int(r.status), r.lower, r.upper, int(r.iterations), x)
        if want_dual:
            return out, y[:2 * self.m].reshape(-1, 2)
        return out

    def launches(self) -> int:
        return int(self._lib.reform_praq_launches(self._h))

    #: kernel kinds of `run_profiled`, in the order the C ABI reports them
    KINDS = ("node", "edge", "node_check", "edge_check", "lower", "check",
             "restart_node", "restart_edge", "restart_check", "mega_block")

    def set_trace(self, capacity: int) -> None:
        """Later runs record every convergence check (iteration, gap, error,
        omega, bounds, restart decision) into a device ring of `capacity`
        records; 0 turns it off."""
        st = self._lib.reform_praq_set_trace(self._h, int(capacity))
        if st != 0:
            raise RuntimeError(f"reform_praq_set_trace failed with status {st}")
        self._trace_ring = max(int(capacity), 0)

    def trace(self, capacity: int = 1 << 16):
        """The last run's checks, oldest first (a NumPy record array with the
        fields of reform_trace_record)."""
        return _native.read_trace(self._lib.reform_praq_trace, self._h, getattr(self, "_trace_ring", 0), capacity)

    def set_megakernel(self, mode: int = -1) -> int:
        """-1: automatic, 0: the per-kernel graph, 1: the persistent kernel's
        single-CTA form where the instance fits, else its grid form, 2: the
        grid form.  Returns the form later runs take: 0 the graph, 1 the grid
        form, 2 the single-CTA form."""
        active = ctypes.c_int(0)
        st = self._lib.reform_praq_set_megakernel(self._h, int(mode), ctypes.byref(active))
        if st != 0:
            raise RuntimeError(f"reform_praq_set_megakernel failed with status {st}")
        return int(active.value)

    def run_profiled(self) -> tuple[int, dict]:
        """A solve with an event pair around every kernel launch; returns the
        status and {kind: (total_ms, launches)}."""
        ms = np.zeros(len(self.KINDS))
        count = np.zeros(len(self.KINDS), dtype=np.int64)
        st = self._lib.reform_praq_run_profiled(self._h, _native.dptr(ms), _native.iptr(count))
        return int(st), {k: (float(ms[i]), int(count[i])) for i, k in enumerate(self.KINDS)}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.reform_praq_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def solve_warm_start(instance, parameters: _native.PraqParameters, warm_start) -> tuple:
    """Solve from a given point, as the reference's solve_qubo_problem_warm_start
    (qubo/praq-jax/praq/solver.py:482-560): `warm_start` = (x, y), x [n] and
    dual pairs y [m, 2] in instance units, both projected before use.  Returns
    (primal [n], dual [m, 2] in instance units, iterations)."""
    with DeviceSolver(instance, parameters) as dev:
        dev.set_warm(*warm_start)
        code = dev.run()
        if code < 0:
            raise RuntimeError(f"reform_praq_run failed with status {code}")
        res, y = dev.result(want_x=True, want_dual=True)
    return res.x, y, res.iterations


def relaxation_bounds(instance, primal, dual) -> tuple[float, float]:
    """(lower, upper) bracket of the relaxation value from a feasible
    primal-dual pair, in instance units (qubo/praq-jax/praq/solver.py:348-362):
    lower = L_D(dual), upper = F(primal).  Evaluated on the device by the
    solver's own bound kernels at the pair (the check before the first step of
    a solve started there); the pair is projected first, which leaves a
    feasible pair as it is."""
    p = _native.lib().praq_default_parameters()
    p.tolerance = math.inf      # the check at the start point ends the run
    with DeviceSolver(instance, p) as dev:
        dev.set_warm(primal, dual)
        code = dev.run()
        if code < 0:
            raise RuntimeError(f"reform_praq_run failed with status {code}")
        res = dev.result(want_x=False)
    return res.lower, res.upper


def persistent_variables(primal, tolerance: float = 1e-6) -> tuple[np.ndarray, np.ndarray]:
    """The coordinates a relaxation optimum fixes by persistency of the roof
    dual, and their values (qubo/praq-jax/praq/solver.py:592-611): (mask of
    coordinates within `tolerance` of 0 or 1, rounded values)."""
    x = np.asarray(primal, dtype=np.float64)
    rounded = np.round(x)
    return np.abs(x - rounded) <= tolerance, rounded


def solve(instance, *, tolerances: Tolerances = Tolerances(), time_limit: float = math.inf,
          sample_memory: bool = False, precision: str = "fp64", max_iter: int | None = None,
          **schedule) -> QuboResult:
    """Solve the roof-dual relaxation of `instance` on the GPU.

    The contract of the reference backend: only `tolerances.optimality` reaches
    the solver, as the relative duality gap it stops on; `feasibility` stays
    NaN in the record.  `time_limit` is a wall-clock budget checked between two
    convergence checks (status "time_limit", with the bracket of the last
    check).  `precision` is "fp64" or "mixed" (FP32 iterates, FP64 reductions
    and bounds).  `schedule` overrides fields of `SCHEDULE`.  `sample_memory`
    is accepted for signature compatibility; the device footprint is the
    solver's own allocation and is not sampled.
    """
    common = dict(backend="praq-b200", instance=instance.name, family=instance.family,
                  n=int(instance.n), edges=int(np.asarray(instance.vals).size),
                  optimality_tolerance=tolerances.optimality)
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
    unknown = set(schedule) - set(SCHEDULE)
    if unknown:
        raise KeyError(f"not schedule fields: {sorted(unknown)}")
    lib = Library()
    p = lib.parameters(tolerance=tolerances.optimality, use_float32=int(precision == "mixed"),
                       max_iter=-1 if max_iter is None else int(max_iter), **schedule)
    start = time.perf_counter()
    try:
        solver = DeviceSolver(instance, p)
    except RuntimeError as error:
        return QuboResult(status="error", note=str(error)[:200], **common)
    setup = time.perf_counter() - start
    try:
        if math.isfinite(time_limit):
            solver.set_time_limit(max(0.0, time_limit - setup))
        start = time.perf_counter()
        code = solver.run()
        res = solver.result(want_x=True)
        seconds = time.perf_counter() - start
    finally:
        solver.close()
    if code < 0:
        return QuboResult(status="error", note=f"status {code}", setup_seconds=setup, **common)
    status = STATUS.get(code, "error")
    timed = dict(iterations=res.iterations, setup_seconds=setup, solve_seconds=seconds, **common)
    if status != "optimal":
        return QuboResult(status=status, lower=res.lower, upper=res.upper,
                          note=f"status {code}, relative gap {res.gap:.3g}", **timed)
    return QuboResult(status=status, objective=res.upper, lower=res.lower, upper=res.upper,
                      note=f"precision {precision}", **timed)
