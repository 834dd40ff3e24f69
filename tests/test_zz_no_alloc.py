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
