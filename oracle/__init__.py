"""CPU oracles for the PRAQ and PRIA hot path -- TEST INFRASTRUCTURE ONLY.

Only `tests/`, `__graft_entry__.smoke()` and `bench.py`'s CPU legs may import
this package, and only as the checker or the timed CPU baseline.  The product
(`reformulation_b200`) never imports it.

* `praq_solve` -- our C restatement of PRAQ on the sparse half-edge set
  (oracle/praq_oracle.c; it cites the reference lines it follows).
* `pria_solve` -- our C restatement of PRIA (oracle/pria_oracle.c).
* `ref_pria_solve` -- the reference's own CPU PRIA, `ref::solve` of
  jrp/pria-cuda/tests/ref_impl.hpp, compiled in place into oracle/_ref.
* `ref_praq_solve` -- the reference's own praq-cuda (qubo/praq-cuda/src),
  compiled in place at sm_100a into oracle/_ref; needs a GPU.
* `roof_dual_maxflow` -- the roof dual as a maximum flow on the implication
  network of the QUBO's posiform (Hammer, Hansen and Simeone 1984; Boros and
  Hammer 2002, section 4), our own construction, solved by scipy's
  `maximum_flow` with int32 capacities.
* `half_integral_optimum` -- min of F over {0, 1/2, 1}^n by enumeration, the
  relaxation optimum by half-integrality (n <= 10).
"""

from __future__ import annotations

import ctypes
import itertools
import os
from ctypes import POINTER, c_double, c_int, c_int64
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build" / "liboracle.so"
REF_PRIA = HERE / "_ref" / "libpria_ref.so"
REF_PRAQ = HERE / "_ref" / "libpraq_ref.so"


class OracleParams(ctypes.Structure):
    """The reference's PraqParameters layout (qubo/praq-cuda/include/praq/praq.h:29-60)."""

    _fields_ = [("tolerance", c_double), ("max_iter", c_int64), ("use_float32", c_int),
                ("omega", c_double), ("beta_sufficient", c_double),
                ("beta_necessary", c_double), ("beta_artificial", c_double),
                ("theta_initial", c_double), ("theta_target", c_double),
                ("theta_decay", c_double), ("op_steps", c_int64),
                ("interval_offset", c_double), ("interval_scale", c_double),
                ("interval_power", c_double)]


class OraclePriaParams(ctypes.Structure):
    """The reference's pria_params layout (jrp/pria-cuda/include/pria/pria.h:34-49)."""

    _fields_ = [("omega", c_double), ("eta", c_double), ("beta_sufficient", c_double),
                ("beta_artificial", c_double), ("beta_necessary", c_double),
                ("theta_initial", c_double), ("theta_target", c_double),
                ("theta_decay", c_double), ("tolerance", c_double), ("max_iter", c_int64),
                ("use_halpern", c_int), ("warm_steps", c_int), ("op_steps", c_int),
                ("verbose", c_int)]


def praq_params(**overrides) -> OracleParams:
    """Defaults of Parameters.with_auto_step (qubo/praq-jax/praq/solver.py:129-164)."""
    p = OracleParams(1e-8, -1, 0, 1.0, float(np.exp(-1.0)), 0.5706, 0.2468, 0.81930,
                     0.42818, 0.90474, 16, 0.0, 4.328085122666891, 0.0)
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def pria_params(max_iter: int = -1, tolerance: float = 1e-8, **overrides) -> OraclePriaParams:
    """Defaults of Parameters.with_auto_step (jrp/pria-jax/pria/solver.py:150-188)."""
    p = OraclePriaParams(0.10835, 0.999 / np.sqrt(2.0), float(np.exp(-1.0)), 0.2468, 0.5706,
                         0.81930, 0.42818, 0.90474, tolerance, max_iter, 1, 0, 16, 0)
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


_lib = None


def _oracle():
    global _lib
    if _lib is None:
        if not BUILD.exists():
            raise RuntimeError(f"{BUILD} not built; run `make -C oracle`")
        lib = ctypes.CDLL(str(BUILD))
        lib.oracle_praq_solve.restype = c_int
        lib.oracle_praq_solve.argtypes = [c_int64, c_int64, POINTER(c_double), POINTER(c_int64),
                                          POINTER(c_int64), POINTER(c_double),
                                          POINTER(OracleParams), c_int, POINTER(c_double),
                                          POINTER(c_double), POINTER(c_double)]
        lib.oracle_check_interval.restype = c_int64
        lib.oracle_check_interval.argtypes = [c_int64, c_double, c_double, c_double]
        lib.oracle_praq_relaxation_value.restype = c_double
        lib.oracle_praq_relaxation_value.argtypes = [c_int64, c_int64, POINTER(c_double),
                                                     POINTER(c_int64), POINTER(c_int64),
                                                     POINTER(c_double), POINTER(c_double)]
        lib.oracle_pria_solve.restype = c_int
        lib.oracle_pria_solve.argtypes = [c_int64, c_int64, POINTER(c_double), c_double,
                                          POINTER(c_double), POINTER(OraclePriaParams), c_int,
                                          POINTER(c_double), POINTER(c_double),
                                          POINTER(c_double), POINTER(c_double)]
        lib.oracle_pria_objective.restype = c_double
        lib.oracle_pria_objective.argtypes = [c_int64, c_int64, POINTER(c_double), c_double,
                                              POINTER(c_double), POINTER(c_double)]
        _lib = lib
    return _lib


def _d(a):
    return a.ctypes.data_as(POINTER(c_double))


def _i(a):
    return a.ctypes.data_as(POINTER(c_int64))


def _qubo_arrays(inst):
    return (np.ascontiguousarray(inst.diag, np.float64), np.ascontiguousarray(inst.rows, np.int64),
            np.ascontiguousarray(inst.cols, np.int64), np.ascontiguousarray(inst.vals, np.float64))


def praq_solve(inst, params: OracleParams | None = None, threads: int = 1, want_dual=False):
    """Solve the roof-dual LP of a QUBO instance with the C restatement.

    Returns a dict: status, lower, upper, iterations, x (and y, the half-edge
    dual pairs in the instance's units, with `want_dual`)."""
    params = params or praq_params()
    diag, rows, cols, vals = _qubo_arrays(inst)
    x = np.empty(inst.n)
    y = np.empty(2 * max(inst.edges, 1)) if want_dual else None
    out = np.empty(4)
    status = _oracle().oracle_praq_solve(inst.n, inst.edges, _d(diag), _i(rows), _i(cols),
                                         _d(vals), ctypes.byref(params), threads, _d(x),
                                         _d(y) if y is not None else None, _d(out))
    res = dict(status=status, lower=out[0], upper=out[1], iterations=int(out[2]), x=x)
    if want_dual:
        res["y"] = y[:2 * inst.edges].reshape(-1, 2)
    return res


def check_interval(n, offset=0.0, scale=4.328085122666891, power=0.0) -> int:
    return int(_oracle().oracle_check_interval(n, offset, scale, power))


def relaxation_value(inst, x) -> float:
    """F(x) of the relaxation, the upper bound at a point, in instance units."""
    diag, rows, cols, vals = _qubo_arrays(inst)
    x = np.ascontiguousarray(x, np.float64)
    return float(_oracle().oracle_praq_relaxation_value(inst.n, inst.edges, _d(diag), _i(rows),
                                                        _i(cols), _d(vals), _d(x)))


def qubo_lower_bound(inst, y_pairs) -> float:
    """L_D(y) (qubo/praq-jax/praq/solver.py:333-337) for half-edge duals in
    instance units: sum_i min(d_i - (S^T y)_i, 0) + sum over covering edges of
    y_e,1.  A valid lower bound whenever y lies in the dual set."""
    y = np.asarray(y_pairs, np.float64).reshape(-1, 2)
    st = np.zeros(inst.n)
    np.add.at(st, inst.rows, y[:, 0])
    np.add.at(st, inst.cols, y[:, 1])
    rc = inst.diag - st
    return float(np.minimum(rc, 0.0).sum() + y[inst.vals > 0, 0].sum())


def half_integral_optimum(inst) -> float:
    """min F(x) over {0, 1/2, 1}^n (n <= 10): the relaxation optimum."""
    if inst.n > 10:
        raise ValueError("enumeration is for n <= 10")
    best = np.inf
    grid = np.array(list(itertools.product((0.0, 0.5, 1.0), repeat=inst.n)))
    xi, xj = grid[:, inst.rows], grid[:, inst.cols]
    w = 2.0 * inst.vals
    edge = np.where(w > 0, w * np.maximum(xi + xj - 1.0, 0.0), w * np.minimum(xi, xj))
    vals = grid @ inst.diag + edge.sum(axis=1)
    best = float(vals.min())
    return best


def roof_dual_maxflow(inst) -> float:
    """The roof dual (= the LP optimum) as constant + max-flow / 2.

    Posiform: x^T W x = sum_i d_i x_i + sum_e c_e x_i x_j with c_e = 2 W_ij.  A
    negative product is rewritten c x_i x_j = c x_i + |c| x_i (1 - x_j), moving
    c onto the linear coefficient of x_i; a negative linear coefficient a
    becomes a + |a| (1 - x_i).  Every remaining term a * u * v (literals u, v;
    a linear term uses the always-true literal) gives two arcs, NOT u -> v and
    NOT v -> u, each of capacity a / 2.  Nodes: literal x_i is 2i, its
    complement 2i + 1, the always-false literal (source) 2n, the always-true
    literal (sink) 2n + 1, so complementing is XOR 1.  Capacities are doubled
    to stay integral (weights here are integers), so the flow is halved.
    """
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import maximum_flow

    n = inst.n
    c = 2.0 * np.asarray(inst.vals, np.float64)
    rows = np.asarray(inst.rows, np.int64)
    cols = np.asarray(inst.cols, np.int64)
    nz = c != 0.0
    c, rows, cols = c[nz], rows[nz], cols[nz]
    lin = np.asarray(inst.diag, np.float64).copy()
    neg = c < 0.0
    np.add.at(lin, rows[neg], c[neg])
    constant = float(lin[lin < 0.0].sum())
    source, sink = 2 * n, 2 * n + 1
    # quadratic terms: u = x_i, v = x_j (positive) or NOT x_j (negative)
    u_q = 2 * rows
    v_q = 2 * cols + neg.astype(np.int64)
    a_q = np.abs(c)
    # linear terms: u = x_i (a >= 0) or NOT x_i (a < 0), v = always-true
    u_l = 2 * np.arange(n, dtype=np.int64) + (lin < 0.0).astype(np.int64)
    v_l = np.full(n, sink, np.int64)
    a_l = np.abs(lin)
    u = np.concatenate([u_q, u_l])
    v = np.concatenate([v_q, v_l])
    a = np.concatenate([a_q, a_l])
    if not np.allclose(a, np.round(a)):
        raise ValueError("integer weights only")
    a = np.round(a).astype(np.int64)
    keep = a > 0
    u, v, a = u[keep], v[keep], a[keep]
    tails = np.concatenate([u ^ 1, v ^ 1])
    heads = np.concatenate([v, u])
    caps = np.concatenate([a, a])
    if caps.sum() >= 2 ** 31:
        raise ValueError("total capacity exceeds int32")
    graph = csr_matrix((caps.astype(np.int32), (tails, heads)), shape=(2 * n + 2, 2 * n + 2))
    graph.sum_duplicates()
    flow = maximum_flow(graph, source, sink, method="dinic").flow_value
    return constant + flow / 2.0


# --- PRIA ---------------------------------------------------------------------

def _jrp_arrays(inst):
    return (np.ascontiguousarray(inst.order_costs, np.float64),
            float(inst.joint_order_cost),
            np.ascontiguousarray(inst.holding_costs, np.float64))


def pria_solve(inst, params: OraclePriaParams | None = None, threads: int = 1,
               want_solution=False):
    """Solve a JRP LP with the C restatement.  Returns iterations, upper
    (primal objective at the unpadded x), lower (padded dual bound), gap, and
    x, y, z with `want_solution` (duals normalised by K_i and K0)."""
    params = params or pria_params()
    k, k0, h = _jrp_arrays(inst)
    n, t = inst.items, inst.periods
    sol = [np.empty(n * t * t) for _ in range(3)] if want_solution else [None] * 3
    out = np.empty(4)
    _oracle().oracle_pria_solve(n, t, _d(k), k0, _d(h), ctypes.byref(params), threads,
                                *[(_d(a) if a is not None else None) for a in sol], _d(out))
    res = dict(iterations=int(out[0]), upper=out[1], lower=out[2], gap=out[3])
    if want_solution:
        res.update(x=sol[0].reshape(n, t, t), y=sol[1].reshape(n, t, t),
                   z=sol[2].reshape(n, t, t))
    return res


def pria_objective(inst, x) -> float:
    k, k0, h = _jrp_arrays(inst)
    x = np.ascontiguousarray(x, np.float64)
    return float(_oracle().oracle_pria_objective(inst.items, inst.periods, _d(k), k0, _d(h),
                                                 _d(x)))


def pria_dual_bound(inst, y, z) -> float:
    """sum_{i,t} min_{s<=t}(H + K_i y + K0 z) for normalised duals
    (jrp/pria-jax/pria/solver.py:740-790): valid for any feasible pair."""
    h = np.triu(np.asarray(inst.holding_costs, np.float64))
    reduced = h + inst.order_costs[:, None, None] * y + inst.joint_order_cost * z
    t = h.shape[-1]
    per = np.arange(t)
    reduced = np.where(per[:, None] <= per[None, :], reduced, np.inf)
    return float(reduced.min(axis=1).sum())


_ref_pria = None


def ref_pria_available() -> bool:
    return REF_PRIA.exists()


def _ref_pria_lib():
    global _ref_pria
    if _ref_pria is None:
        if not REF_PRIA.exists():
            raise RuntimeError(f"{REF_PRIA} not built; run `make -C oracle ref`")
        lib = ctypes.CDLL(str(REF_PRIA))
        lib.ref_pria_solve.restype = c_int
        lib.ref_pria_solve.argtypes = [c_int64, c_int64, POINTER(c_double), c_double,
                                       POINTER(c_double), POINTER(OraclePriaParams),
                                       POINTER(c_double), POINTER(c_double), POINTER(c_double),
                                       POINTER(c_double)]
        lib.ref_pria_random_instance.restype = None
        lib.ref_pria_random_instance.argtypes = [ctypes.c_uint64, c_int64, c_int64,
                                                 POINTER(c_double), POINTER(c_double),
                                                 POINTER(c_double)]
        _ref_pria = lib
    return _ref_pria


def ref_pria_solve(inst, params: OraclePriaParams | None = None, want_solution=False):
    """The reference's own CPU PRIA (ref::solve), FP64, one core."""
    lib = _ref_pria_lib()
    params = params or pria_params()
    k, k0, h = _jrp_arrays(inst)
    n, t = inst.items, inst.periods
    sol = [np.empty(n * t * t) for _ in range(3)] if want_solution else [None] * 3
    out = np.empty(4)
    lib.ref_pria_solve(n, t, _d(k), k0, _d(h), ctypes.byref(params),
                       *[(_d(a) if a is not None else None) for a in sol], _d(out))
    res = dict(iterations=int(out[0]), upper=out[1], lower=out[2], gap=out[3])
    if want_solution:
        res.update(x=sol[0].reshape(n, t, t), y=sol[1].reshape(n, t, t),
                   z=sol[2].reshape(n, t, t))
    return res


def ref_pria_random_instance(seed: int, n: int, t: int):
    """ref::random_instance of the reference's CUDA tests, as a JrpInstance."""
    from reformulation_b200.instances import JrpInstance
    lib = _ref_pria_lib()
    k = np.empty(n)
    k0 = np.empty(1)
    h = np.empty(n * t * t)
    lib.ref_pria_random_instance(seed, n, t, _d(k), _d(k0), _d(h))
    return JrpInstance(f"ref-random-n{n}-t{t}-s{seed}", "ref-random", k, float(k0[0]),
                       h.reshape(n, t, t))


class RefPraq:
    """The reference's praq-cuda library (praq_solve), built at sm_100a.  GPU only."""

    def __init__(self):
        if not REF_PRAQ.exists():
            raise RuntimeError(f"{REF_PRAQ} not built; run `make -C oracle ref`")
        self.lib = ctypes.CDLL(str(REF_PRAQ))
        self.lib.praq_default_parameters.restype = OracleParams
        self.lib.praq_solve.restype = c_int

    def solve(self, inst, tolerance=1e-8, use_float32=0, max_iter=-1):
        class Inst(ctypes.Structure):
            _fields_ = [("n", c_int64), ("m", c_int64), ("diag", POINTER(c_double)),
                        ("rows", POINTER(c_int64)), ("cols", POINTER(c_int64)),
                        ("vals", POINTER(c_double))]

        class Res(ctypes.Structure):
            _fields_ = [("lower", c_double), ("upper", c_double), ("iterations", c_int64),
                        ("status", c_int)]

        diag, rows, cols, vals = _qubo_arrays(inst)
        view = Inst(inst.n, inst.edges, _d(diag), _i(rows), _i(cols), _d(vals))
        p = self.lib.praq_default_parameters()
        p.tolerance, p.use_float32, p.max_iter = tolerance, use_float32, max_iter
        x = np.empty(inst.n)
        r = Res()
        st = self.lib.praq_solve(ctypes.byref(view), ctypes.byref(p), _d(x), ctypes.byref(r))
        return dict(status=st, lower=r.lower, upper=r.upper, iterations=int(r.iterations), x=x)


def threads_available() -> int:
    return len(os.sched_getaffinity(0))
