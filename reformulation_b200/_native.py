"""ctypes binding of libreform_b200.so, the C ABI declared in include/*.h.

There is no fallback: if the library is missing or fails to load, every solve
raises.  The structs mirror the headers field for field (the PRAQ and PRIA ones
are byte-compatible with the reference's praq.h / pria.h).
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_int64, c_void_p
from pathlib import Path

import numpy as np

# REFORM_B200_LIB names another build of the library (the checked build,
# libreform_b200_debug_bounds.so); the default is the in-tree release build.
LIB_PATH = Path(os.environ.get("REFORM_B200_LIB") or Path(__file__).resolve().parent / "_lib" / "libreform_b200.so")


class PraqInstance(ctypes.Structure):
    _fields_ = [("n", c_int64), ("m", c_int64), ("diag", POINTER(c_double)),
                ("rows", POINTER(c_int64)), ("cols", POINTER(c_int64)),
                ("vals", POINTER(c_double))]


class PraqParameters(ctypes.Structure):
    _fields_ = [("tolerance", c_double), ("max_iter", c_int64), ("use_float32", c_int),
                ("omega", c_double), ("beta_sufficient", c_double),
                ("beta_necessary", c_double), ("beta_artificial", c_double),
                ("theta_initial", c_double), ("theta_target", c_double),
                ("theta_decay", c_double), ("op_steps", c_int64),
                ("interval_offset", c_double), ("interval_scale", c_double),
                ("interval_power", c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PraqResult(ctypes.Structure):
    _fields_ = [("lower", c_double), ("upper", c_double), ("iterations", c_int64),
                ("status", c_int)]


class PriaParams(ctypes.Structure):
    _fields_ = [("omega", c_double), ("eta", c_double), ("beta_sufficient", c_double),
                ("beta_artificial", c_double), ("beta_necessary", c_double),
                ("theta_initial", c_double), ("theta_target", c_double),
                ("theta_decay", c_double), ("tolerance", c_double), ("max_iter", c_int64),
                ("use_halpern", c_int), ("warm_steps", c_int), ("op_steps", c_int),
                ("verbose", c_int)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PriaResultInfo(ctypes.Structure):
    _fields_ = [("iterations", c_int64), ("primal_objective", c_double),
                ("dual_objective", c_double), ("relative_gap", c_double)]


class ReformShapes(ctypes.Structure):
    _fields_ = [("reserved0", c_int), ("grid_multiplier", c_int),
                ("reserved", c_int * 6)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("budget_bytes", c_int64), ("tolerance", c_double), ("max_iter", c_int64),
                ("use_float32", c_int), ("blocks_in_flight", c_int), ("admit_every", c_int),
                ("stall_iterations", c_int)]


class ServerRequest(ctypes.Structure):
    _fields_ = [("state", c_int), ("error", c_int), ("kind", c_int), ("escalated", c_int),
                ("iterations", c_int64), ("lower", c_double), ("upper", c_double),
                ("arrival", c_double), ("admitted", c_double), ("finished", c_double),
                ("device_bytes", c_int64)]


class ServerCounts(ctypes.Structure):
    _fields_ = [("waiting", c_int64), ("running", c_int64), ("completed", c_int64),
                ("reserved_bytes", c_int64), ("high_water_bytes", c_int64),
                ("device_bytes", c_int64), ("error", c_int)]


_lib = None


def _declare(lib):
    D, I, L = POINTER(c_double), c_int, c_int64
    P = ctypes.POINTER
    sig = {
        "praq_default_parameters": (PraqParameters, []),
        "praq_check_interval": (c_int64, [c_int64, P(PraqParameters)]),
        "praq_solve": (I, [P(PraqInstance), P(PraqParameters), D, P(PraqResult)]),
        "reform_praq_create": (I, [P(PraqInstance), P(PraqParameters), c_void_p,
                                   P(c_void_p)]),
        "reform_praq_run": (I, [c_void_p]),
        "reform_praq_result": (I, [c_void_p, D, D, P(PraqResult)]),
        "reform_praq_set_time_limit": (I, [c_void_p, c_double]),
        "reform_praq_set_warm": (I, [c_void_p, P(c_double), P(c_double)]),
        "reform_praq_run_profiled": (I, [c_void_p, D, P(c_int64)]),
        "reform_praq_set_megakernel": (I, [c_void_p, c_int, P(c_int)]),
        "reform_praq_set_trace": (I, [c_void_p, c_int]),
        "reform_praq_trace": (I, [c_void_p, c_void_p, c_int, P(c_int64)]),
        "reform_pria_set_trace": (I, [c_void_p, c_int]),
        "reform_pria_trace": (I, [c_void_p, c_void_p, c_int, P(c_int64)]),
        "reform_praq_launches": (c_int64, [c_void_p]),
        "reform_praq_destroy": (None, [c_void_p]),
        "reform_praq_bounds_noalloc": (I, [c_int64, c_int64, c_void_p, c_void_p, c_void_p,
                                           c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    }
    F = POINTER(ctypes.c_float)
    sig.update({
        "pria_params_auto": (PriaParams, [c_int64, c_double]),
        "pria_solve_f64": (I, [c_int64, c_int64, D, c_double, D, P(PriaParams), D, D, D, D, D, D,
                               P(PriaResultInfo)]),
        "pria_solve_f32": (I, [c_int64, c_int64, F, ctypes.c_float, F, P(PriaParams), F, F, F, F, F,
                               F, P(PriaResultInfo)]),
        "pria_solve_batch_f64": (I, [c_int64, c_int64, c_int64, D, D, D, P(PriaParams), D, D, D,
                                     P(PriaResultInfo)]),
        "pria_solve_batch_f32": (I, [c_int64, c_int64, c_int64, F, F, F, P(PriaParams), F, F, F,
                                     P(PriaResultInfo)]),
        "pria_objective_f64": (c_double, [c_int64, c_int64, D, c_double, D, D]),
        "reform_pria_create": (I, [c_int64, c_int64, D, c_double, D, P(PriaParams), I, c_void_p,
                                   P(c_void_p)]),
        "reform_pria_run": (I, [c_void_p]),
        "reform_pria_set_time_limit": (I, [c_void_p, c_double]),
        "reform_pria_set_warm": (I, [c_void_p, D, D, D]),
        "reform_pria_result": (I, [c_void_p, D, D, D, P(PriaResultInfo)]),
        "reform_pria_run_profiled": (I, [c_void_p, D, P(c_int64)]),
        "reform_pria_set_megakernel": (I, [c_void_p, c_int, P(c_int)]),
        "reform_pria_launches": (c_int64, [c_void_p]),
        "reform_pria_destroy": (None, [c_void_p]),
    })
    V = c_void_p
    sig.update({
        "reform_batch_create": (I, [I, V, P(V)]),
        "reform_batch_add_qubo": (I, [V, P(PraqInstance), P(PraqParameters)]),
        "reform_batch_add_jrp": (I, [V, c_int64, c_int64, D, c_double, D, P(PriaParams)]),
        "reform_batch_add_jrp_demand": (I, [V, c_int64, c_int64, D, c_double, D, D, P(PriaParams)]),
        "reform_batch_start": (I, [V]),
        "reform_batch_run": (I, [V, c_int64]),
        "reform_batch_launch": (I, [V]),
        "reform_batch_sync": (I, [V, P(c_int), I, P(c_int)]),
        "reform_batch_inflight": (I, [V]),
        "reform_batch_status": (I, [V, I, P(c_int), P(c_int64), D, D]),
        "reform_batch_result_qubo": (I, [V, I, D, P(PraqResult)]),
        "reform_batch_result_jrp": (I, [V, I, D, D, D, P(PriaResultInfo)]),
        "reform_batch_remove": (I, [V, I]),
        "reform_batch_set_warm_qubo": (I, [V, I, D, D]),
        "reform_batch_point_qubo": (I, [V, I, D, D]),
        "reform_batch_device_bytes": (c_int64, [V]),
        "reform_batch_set_shapes": (I, [V, P(ReformShapes)]),
        "reform_batch_autotune": (I, [V, P(ReformShapes)]),
        "reform_batch_restart": (I, [V]),
        "reform_batch_launches": (c_int64, [V]),
        "reform_batch_destroy": (None, [V]),
        "reform_server_default_options": (ServerOptions, []),
        "reform_server_create": (I, [P(ServerOptions), P(V)]),
        "reform_server_submit_qubo": (c_int64, [V, P(PraqInstance)]),
        "reform_server_submit_jrp": (c_int64, [V, c_int64, c_int64, D, c_double, D]),
        "reform_server_submit_jrp_demand": (c_int64, [V, c_int64, c_int64, D, c_double, D, D]),
        "reform_server_poll": (I, [V, P(c_int64), I, P(c_int), c_double]),
        "reform_server_status": (I, [V, c_int64, P(ServerRequest)]),
        "reform_server_result_qubo": (I, [V, c_int64, D, P(PraqResult)]),
        "reform_server_result_jrp": (I, [V, c_int64, D, D, D, P(PriaResultInfo)]),
        "reform_server_retire": (I, [V, c_int64]),
        "reform_server_stats": (I, [V, P(ServerCounts)]),
        "reform_server_destroy": (None, [V]),
    })
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


# reform_trace_record (include/reform_trace.h), as a NumPy record type
TRACE_DTYPE = np.dtype([("iteration", np.int64), ("gap", np.float64), ("error", np.float64),
                        ("omega", np.float64), ("lower", np.float64), ("upper", np.float64),
                        ("restart", np.int32), ("terminated", np.int32)])


def read_trace(fn, handle, ring: int, capacity: int = 1 << 16):
    """The last run's convergence trace through `fn` (reform_praq_trace or
    reform_pria_trace) from a ring of `ring` records, oldest first, as a
    TRACE_DTYPE array."""
    total = c_int64(0)
    out = np.zeros(capacity, TRACE_DTYPE)
    st = fn(handle, out.ctypes.data_as(c_void_p), capacity, ctypes.byref(total))
    if st != 0:
        raise RuntimeError(f"reading the trace failed with status {st}")
    return out[:min(int(total.value), ring, capacity)].copy()


def lib():
    """The loaded native library; raises if it is absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is not built; run `python -m reformulation_b200.build`. "
                "There is no CPU fallback.")
        _lib = _declare(ctypes.CDLL(str(LIB_PATH)))
    return _lib


def dptr(a):
    return a.ctypes.data_as(POINTER(c_double))


def fptr(a):
    return a.ctypes.data_as(POINTER(ctypes.c_float))


def iptr(a):
    return a.ctypes.data_as(POINTER(c_int64))
