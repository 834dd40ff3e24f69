"""reform_praq_bounds_noalloc: the roof-dual bracket of a point computed with
no device allocation (its scratch is a fixed array inside the library), for
callers that may not allocate device memory where they need a certificate --
inside their own stream capture, in allocator-free real-time loops, or inside a
framework that owns all device memory.

Checked through the C ABI against the existing entry point: the bracket
reform_praq_run / reform_praq_result report for the same solve, within 1e-9
relative (the solver keeps FP64 iterates in scaled units, this entry point sums
the same point in instance units), on two calls in a row (the scratch keeps the
last call's contents, so the second call shows it clears what it must).  The
caller-side device buffers are allocated by the test (torch), never by the
entry point.  This file is collected last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def _device(t):
    import torch
    return torch.from_numpy(np.ascontiguousarray(t)).cuda()


@pytest.mark.parametrize("which", ["bernoulli-n200", "uniform-n3000"])
def test_noalloc_bounds_match_solver(native, which):
    import torch

    from reformulation_b200 import _native, praq
    from reformulation_b200.instances import qubo_sparse_bernoulli, qubo_uniform_edges

    inst = (qubo_sparse_bernoulli(0, 200, 0.05) if which == "bernoulli-n200"
            else qubo_uniform_edges(5, 3000, 30000))
    lib = praq.Library()
    with praq.DeviceSolver(inst, lib.parameters(tolerance=1e-9)) as dev:
        assert dev.run() == 0
        res, y = dev.result(want_x=True, want_dual=True)

    args = [_device(a) for a in (inst.diag.astype(np.float64), inst.rows.astype(np.int64),
                                 inst.cols.astype(np.int64), inst.vals.astype(np.float64),
                                 res.x, y.reshape(-1))]
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    L = _native.lib()
    for _ in range(2):
        out.fill_(float("nan"))
        rc = L.reform_praq_bounds_noalloc(inst.n, inst.edges, *[a.data_ptr() for a in args],
                                          out.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        lower, upper = out.tolist()
        assert rel(lower, res.lower) <= 1e-9, (lower, res.lower)
        assert rel(upper, res.upper) <= 1e-9, (upper, res.upper)


def test_noalloc_rejects_beyond_its_scratch(native):
    import torch

    from reformulation_b200 import _native
    L = _native.lib()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    # n above the fixed maximum (262,144 nodes) is refused before any launch
    assert L.reform_praq_bounds_noalloc(262_145, 0, p, None, None, None, p, None, p, None) == -2
    assert L.reform_praq_bounds_noalloc(0, 0, p, None, None, None, p, None, p, None) == -2
    assert L.reform_praq_bounds_noalloc(4, 0, None, None, None, None, p, None, p, None) == -1


def _bracket(inst, x, y):
    """The entry point on device copies of (instance, x, y): (rc, lower, upper)."""
    import torch

    from reformulation_b200 import _native
    args = [_device(a) for a in (np.asarray(inst.diag, np.float64), np.asarray(inst.rows, np.int64),
                                 np.asarray(inst.cols, np.int64), np.asarray(inst.vals, np.float64),
                                 np.asarray(x, np.float64), np.asarray(y, np.float64).reshape(-1))]
    if inst.edges == 0:      # an empty tensor may have no address: pass a valid one
        args[1] = args[2] = _device(np.zeros(1, np.int64))
        args[3] = args[5] = _device(np.zeros(2))
    out = torch.full((2,), 7.0, dtype=torch.float64, device="cuda")
    rc = _native.lib().reform_praq_bounds_noalloc(inst.n, inst.edges, *[a.data_ptr() for a in args],
                                                  out.data_ptr(),
                                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    lower, upper = out.tolist()
    return rc, lower, upper


def test_noalloc_bad_edges_give_nan(native):
    """An edge index out of range, or a self-loop, is flagged on the device:
    both outputs are NaN; the next valid call is unaffected."""
    from reformulation_b200.instances import QuboInstance
    rng = np.random.default_rng(2)
    n = 50
    rows, cols = rng.integers(0, n, 40), rng.integers(0, n, 40)
    rows, cols = np.minimum(rows, cols), np.maximum(rows, cols)
    keep = rows != cols
    base = QuboInstance("b", "b", n, rng.normal(size=n), rows[keep], cols[keep],
                        rng.normal(size=keep.sum()))
    x, y = rng.uniform(0, 1, n), rng.normal(size=(base.edges, 2))
    for bad_col in (n, -1, int(base.rows[3])):      # past the end, negative, a self-loop
        c = base.cols.copy()
        c[3] = bad_col
        bad = QuboInstance("x", "x", n, base.diag, base.rows, c, base.vals)
        rc, lower, upper = _bracket(bad, x, y)
        assert rc == 0 and np.isnan(lower) and np.isnan(upper), bad_col
    rc, lower, upper = _bracket(base, x, y)
    assert rc == 0 and np.isfinite(lower) and np.isfinite(upper)


def test_noalloc_without_edges(native):
    """m = 0: the node pass alone, lower = sum min(d, 0) and upper = d.x."""
    from reformulation_b200.instances import QuboInstance
    rng = np.random.default_rng(3)
    n = 1000
    inst = QuboInstance("e", "e", n, rng.normal(size=n), np.zeros(0, np.int64), np.zeros(0, np.int64),
                        np.zeros(0))
    x = rng.uniform(0, 1, n)
    rc, lower, upper = _bracket(inst, x, np.zeros(0))
    assert rc == 0
    assert rel(lower, np.minimum(inst.diag, 0).sum()) <= 1e-12
    assert rel(upper, inst.diag @ x) <= 1e-12


def test_noalloc_at_its_largest_instance(native, oracle_lib):
    """n = 262,144, the largest instance the fixed scratch holds (the last
    node's accumulator is its last S^T y slot), against the oracle's bracket
    of the same point."""
    from reformulation_b200.instances import qubo_uniform_edges
    n = 262_144
    inst = qubo_uniform_edges(8, n, 40_000)
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 1, n)
    w = 2.0 * np.abs(inst.vals)
    y = np.where((inst.vals > 0)[:, None], -0.5 * w[:, None], 0.5 * w[:, None]) * np.ones((1, 2))
    # an edge at the very last node, so the scratch boundary is exercised
    rows = np.append(inst.rows, 0)
    cols = np.append(inst.cols, n - 1)
    vals = np.append(inst.vals, -3.0)
    y = np.vstack([y, [3.0, 3.0]])
    from reformulation_b200.instances import QuboInstance
    full = QuboInstance("big", "big", n, inst.diag, rows, cols, vals)
    rc, lower, upper = _bracket(full, x, y)
    assert rc == 0
    assert rel(upper, oracle_lib.relaxation_value(full, x)) <= 1e-12
    assert rel(lower, oracle_lib.qubo_lower_bound(full, y)) <= 1e-12
