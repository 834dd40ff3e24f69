"""PRAQ on the GPU against the oracles, through the C ABI (praq_solve and the
reform_praq_* device-resident API).

Patterned on the reference's own checks (qubo/praq-cuda/tests/test_solver.cu:
122-262 and qubo/praq-jax/tests/test_solver.py:40-135): the enumerated
half-integral optimum on tiny instances, bounds that bracket the optimum under
every iteration cap, FP32 reaching its own accuracy, a larger instance
certifying its own gap, rejection of bad inputs; plus agreement with the CPU
restatement (iterations and bounds) and with the max-flow roof dual.

Tolerances: FP64 bounds agree with the optimum to 1e-7 relative at a 1e-9 gap;
FP64 iteration counts agree with the oracle's exactly on these instances (same
arithmetic, different summation order can move a check by one block, so
+-op_steps is allowed); FP32 ("mixed") objectives agree with the FP64
oracle's to 1e-6 relative at the same 1e-4 gap tolerance.
"""

import numpy as np
import pytest

from reformulation_b200.instances import QuboInstance, qubo_sparse_bernoulli

pytestmark = pytest.mark.gpu


def random_qubo(seed, n, density, magnitude=3):
    rng = np.random.default_rng(seed)
    iu = np.triu_indices(n, 1)
    keep = rng.random(iu[0].size) < density
    vals = rng.integers(1, magnitude + 1, keep.sum()) * rng.choice([-1.0, 1.0], keep.sum())
    diag = rng.integers(1, magnitude + 1, n) * rng.choice([-1.0, 1.0], n)
    return QuboInstance(f"r{seed}", "random", n, diag.astype(float), iu[0][keep], iu[1][keep],
                        vals.astype(float))


@pytest.fixture(scope="module")
def lib(native):
    from reformulation_b200.praq import Library
    return Library()


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("density", [1.0, 0.5, 0.2, 0.0])
def test_enumerated_optimum_fp64(lib, oracle_lib, n, density):
    inst = random_qubo(1000 * n + int(10 * density), n, density)
    opt = oracle_lib.half_integral_optimum(inst)
    s = lib.solve(inst, lib.parameters(tolerance=1e-9))
    assert s.status == 0
    assert s.gap <= 1e-9
    assert s.lower <= opt + 1e-9 * (1 + abs(opt)) and s.upper >= opt - 1e-9 * (1 + abs(opt))
    assert rel(s.upper, opt) <= 1e-7
    assert np.all((s.x >= 0) & (s.x <= 1))
    assert abs(oracle_lib.relaxation_value(inst, s.x) - s.upper) <= 1e-9 * (1 + abs(opt))


def test_matches_oracle_config_n200(lib, oracle_lib):
    inst = qubo_sparse_bernoulli(0, 200, 0.05)
    ref = oracle_lib.praq_solve(inst, oracle_lib.praq_params(tolerance=1e-9))
    s = lib.solve(inst, lib.parameters(tolerance=1e-9))
    assert s.status == 0 and ref["status"] == 0
    assert abs(s.iterations - ref["iterations"]) <= 16
    assert rel(s.upper, ref["upper"]) <= 1e-8 and rel(s.lower, ref["lower"]) <= 1e-8
    flow = oracle_lib.roof_dual_maxflow(inst)
    assert rel(s.upper, flow) <= 1e-7 and s.lower <= flow + 1e-6


def test_bounds_bracket_under_every_cap(lib, oracle_lib):
    inst = random_qubo(101, 8, 0.6)
    opt = oracle_lib.half_integral_optimum(inst)
    for cap in (1, 4, 16, 64, 256):
        s = lib.solve(inst, lib.parameters(tolerance=1e-12, max_iter=cap))
        assert s.status in (0, 1)
        assert s.iterations <= cap + 15
        assert s.lower <= opt + 1e-9 * (1 + abs(opt))
        assert s.upper >= opt - 1e-9 * (1 + abs(opt))
        assert s.status == 1 or s.gap <= 1e-12


@pytest.mark.parametrize("n", [4, 6, 8])
def test_float32_accuracy(lib, oracle_lib, n):
    """FP32 iterates: the objective within 1e-6 relative of the FP64 oracle's
    at the same 1e-4 gap tolerance, and a bracket of the optimum."""
    inst = random_qubo(200 + n, n, 0.7)
    opt = oracle_lib.half_integral_optimum(inst)
    ref = oracle_lib.praq_solve(inst, oracle_lib.praq_params(tolerance=1e-4))
    s = lib.solve(inst, lib.parameters(tolerance=1e-4, use_float32=1))
    assert s.status == 0 and s.gap <= 1e-4
    assert rel(s.upper, ref["upper"]) <= 1e-6
    assert s.lower <= opt + 1e-7 * (1 + abs(opt)) and s.upper >= opt - 1e-7 * (1 + abs(opt))


def test_larger_instance_certifies_itself(lib, oracle_lib):
    inst = random_qubo(300, 400, 0.05)
    s = lib.solve(inst, lib.parameters(tolerance=1e-8))
    assert s.status == 0 and s.gap <= 1e-8
    f = oracle_lib.relaxation_value(inst, s.x)
    assert abs(f - s.upper) <= 1e-9 * (1 + abs(f))
    ref = oracle_lib.praq_solve(inst, oracle_lib.praq_params(tolerance=1e-8))
    assert abs(s.iterations - ref["iterations"]) <= 16
    assert rel(s.upper, ref["upper"]) <= 1e-7


def test_dual_certificate_recomputed_on_host(native, oracle_lib):
    from reformulation_b200.praq import DeviceSolver, Library
    inst = qubo_sparse_bernoulli(0, 200, 0.05)
    p = Library().parameters(tolerance=1e-8)
    with DeviceSolver(inst, p) as dev:
        assert dev.run() == 0
        res, y = dev.result(want_x=True, want_dual=True)
    # dual feasibility (covering: equal pair in [-w, 0]; packing: a + b = w, both >= 0)
    w = 2.0 * np.abs(inst.vals)
    cov = inst.vals > 0
    assert np.all(np.abs(y[cov, 0] - y[cov, 1]) <= 1e-9 * (1 + w[cov]))
    assert np.all(y[cov, 0] <= 1e-12) and np.all(y[cov, 0] >= -w[cov] - 1e-9)
    assert np.all(np.abs(y[~cov].sum(1) - w[~cov]) <= 1e-9 * (1 + w[~cov]))
    assert np.all(y[~cov] >= -1e-12)
    low = oracle_lib.qubo_lower_bound(inst, y)
    assert rel(low, res.lower) <= 1e-9
    assert rel(oracle_lib.relaxation_value(inst, res.x), res.upper) <= 1e-9


def test_deterministic_across_runs(native):
    from reformulation_b200.praq import DeviceSolver, Library
    inst = random_qubo(7, 300, 0.1)
    p = Library().parameters(tolerance=1e-8)
    with DeviceSolver(inst, p) as dev:
        dev.run()
        a = dev.result()
        dev.run()
        b = dev.result()
    assert a.iterations == b.iterations
    assert a.lower == b.lower and a.upper == b.upper
    assert np.array_equal(a.x, b.x)


def test_rejects_bad_input(lib):
    from reformulation_b200 import _native
    import ctypes
    inst = random_qubo(1, 3, 1.0)
    p = lib.parameters()
    x = np.empty(3)
    r = _native.PraqResult()
    L = _native.lib()
    assert L.praq_solve(None, ctypes.byref(p), _native.dptr(x), ctypes.byref(r)) == -1
    bad = QuboInstance("b", "b", 3, inst.diag, inst.rows.copy(), inst.cols.copy(), inst.vals)
    bad.cols[0] = bad.rows[0]
    assert lib.solve(bad, p).status == -2
    bad2 = QuboInstance("b", "b", 3, inst.diag, inst.rows.copy(), inst.cols.copy(), inst.vals)
    bad2.cols[0] = 3
    assert lib.solve(bad2, p).status == -2
    # ends that wrap to valid int32 values must still be rejected
    for v in (-1, (1 << 32) + 1, (1 << 31) + 2, -(1 << 32) + 2):
        bad3 = QuboInstance("b", "b", 3, inst.diag, inst.rows.copy(), inst.cols.copy(), inst.vals)
        bad3.rows[1] = v
        assert lib.solve(bad3, p).status == -2
    empty = QuboInstance("e", "e", 0, np.zeros(0), np.zeros(0, np.int64), np.zeros(0, np.int64),
                         np.zeros(0))
    assert lib.solve(empty, p).status == -2
    q = lib.parameters(omega=-1.0)
    assert lib.solve(inst, q).status == -1


def test_interval_rule_op_steps_zero(lib):
    p = lib.parameters()
    assert lib.check_interval(50_000, lib.parameters(op_steps=0)) == 2
    inst = random_qubo(3, 60, 1.0)
    s = lib.solve(inst, lib.parameters(tolerance=1e-8, op_steps=0))
    assert s.status == 0
    assert s.iterations % 2 == 0 and s.iterations > 0
    del p


def test_backend_solve_api(native):
    from reformulation_b200 import praq
    from reformulation_b200.results import Tolerances
    inst = qubo_sparse_bernoulli(0, 200, 0.05)
    r = praq.solve(inst, tolerances=Tolerances(optimality=1e-6), time_limit=60.0)
    assert r.status == "optimal" and r.objective == r.upper
    assert r.iterations > 0 and np.isnan(r.feasibility_tolerance)
    m = praq.solve(inst, tolerances=Tolerances(optimality=1e-4), time_limit=60.0,
                   precision="mixed")
    f = praq.solve(inst, tolerances=Tolerances(optimality=1e-4), time_limit=60.0)
    assert m.status == "optimal" and f.status == "optimal"
    assert rel(m.objective, f.objective) <= 1e-6
    c = praq.solve(inst, tolerances=Tolerances(optimality=1e-12), time_limit=60.0, max_iter=32)
    assert c.status == "iteration_limit" and np.isnan(c.objective) and c.lower <= c.upper


def test_unsorted_and_reversed_edges(lib, oracle_lib):
    """Edges in any order and either orientation: the device layout sorts
    them; the optimum and the returned primal do not depend on the order."""
    inst = qubo_sparse_bernoulli(0, 200, 0.05)
    rng = np.random.default_rng(9)
    order = rng.permutation(inst.edges)
    flip = rng.random(inst.edges) < 0.5
    rows, cols = inst.rows[order].copy(), inst.cols[order].copy()
    rows[flip], cols[flip] = cols[flip], rows[flip].copy()
    shuffled = QuboInstance("s", "s", inst.n, inst.diag, rows, cols, inst.vals[order])
    a = lib.solve(inst, lib.parameters(tolerance=1e-9))
    b = lib.solve(shuffled, lib.parameters(tolerance=1e-9))
    flow = oracle_lib.roof_dual_maxflow(inst)
    assert a.status == 0 and b.status == 0
    assert rel(a.upper, flow) <= 1e-7 and rel(b.upper, flow) <= 1e-7
    assert abs(oracle_lib.relaxation_value(inst, b.x) - b.upper) <= 1e-9 * (1 + abs(flow))
    from reformulation_b200.praq import DeviceSolver
    with DeviceSolver(shuffled, lib.parameters(tolerance=1e-8)) as dev:
        dev.run()
        res, y = dev.result(want_dual=True)
    low = oracle_lib.qubo_lower_bound(shuffled, y)
    assert rel(low, res.lower) <= 1e-9


def test_warm_start_and_relaxation_bounds(native, oracle_lib):
    """The warm-start API of qubo/praq-jax/praq/solver.py:482-560: from the
    optimum it ends at the check before the first step; from any point
    (projected) it reaches the same optimum.  relaxation_bounds at the
    returned pair is the bracket the solver reported (solver.py:348-362)."""
    from reformulation_b200 import praq
    inst = qubo_sparse_bernoulli(0, 200, 0.05)
    lib = praq.Library()
    p = lib.parameters(tolerance=1e-9)
    with praq.DeviceSolver(inst, p) as dev:
        assert dev.run() == 0
        cold, y = dev.result(want_x=True, want_dual=True)
    lo, up = praq.relaxation_bounds(inst, cold.x, y)
    assert rel(lo, cold.lower) <= 1e-12 and rel(up, cold.upper) <= 1e-12
    x, y2, its = praq.solve_warm_start(inst, p, (cold.x, y))
    assert its == 0 and np.array_equal(x, cold.x)
    rng = np.random.default_rng(3)
    far = (rng.uniform(-1, 2, inst.n), rng.normal(0, 50, (inst.edges, 2)))
    x, y2, its = praq.solve_warm_start(inst, p, far)
    lo, up = praq.relaxation_bounds(inst, x, y2)
    flow = oracle_lib.roof_dual_maxflow(inst)
    assert its > 0 and lo <= flow + 1e-7 * (1 + abs(flow)) <= up + 2e-7 * (1 + abs(flow))
    assert rel(up, flow) <= 1e-7
    assert np.all((x >= 0) & (x <= 1))
    fixed, vals = praq.persistent_variables(x)
    assert fixed.any() and set(np.unique(vals[fixed])) <= {0.0, 1.0}


def test_edgeless_instance_terminates(lib):
    """No edges: the edge partial sums the checks read are zeros (not stale
    pool memory), so the solve ends."""
    inst = QuboInstance("e", "e", 5, np.array([-2.0, 1.0, 3.0, -1.0, 0.0]), np.zeros(0, np.int64),
                        np.zeros(0, np.int64), np.zeros(0))
    for _ in range(3):
        s = lib.solve(inst, lib.parameters(tolerance=1e-9, max_iter=10_000))
        assert s.status == 0 and abs(s.upper - (-3.0)) <= 1e-8


@pytest.mark.parametrize("use_float32", [0, 1])
def test_gated_block_graph(native, use_float32):
    """A solver's first run launches its kernels one by one; later runs
    replay the captured check block, a conditional graph whose body runs only
    while the solve has not terminated.  The results are the first run's bit
    for bit, and the block queued behind the one that ended the solve runs its
    gate kernel alone, so a replayed run launches fewer kernels than the first
    (the same number every time)."""
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.praq import DeviceSolver, Library
    inst = qubo_uniform_edges(5, 20000, 200000)
    p = Library().parameters(tolerance=1e-4 if use_float32 else 1e-7, use_float32=use_float32)
    runs, launches = [], []
    with DeviceSolver(inst, p) as dev:
        dev.set_megakernel(0)
        for _ in range(3):
            assert dev.run() == 0
            runs.append(dev.result(want_x=True, want_dual=True))
            launches.append(dev.launches())
    (a, ya), *rest = runs
    for b, yb in rest:
        assert (a.iterations, a.lower, a.upper) == (b.iterations, b.lower, b.upper)
        assert np.array_equal(a.x, b.x) and np.array_equal(ya, yb)
    assert launches[1] < launches[0] and launches[2] == launches[1], launches


@pytest.mark.parametrize("use_float32", [0, 1])
def test_upload_modes_agree(lib, monkeypatch, use_float32):
    """The instance arrays cross to the device by the driver's copy (the
    default) or through the library's pinned staging ring ("staged"): the
    same layout, so the same solve bit for bit, sorted or shuffled; and both
    reject an end out of range or a self-loop anywhere in the arrays.  25k
    edges: above the size whose flags the set-up finds on the host, so the
    device's scan raises them."""
    base = random_qubo(21, 5000, 0.002)
    assert base.edges > 16384
    rng = np.random.default_rng(3)
    order = rng.permutation(base.edges)
    flip = rng.random(base.edges) < 0.5
    rows, cols = base.rows[order].copy(), base.cols[order].copy()
    rows[flip], cols[flip] = cols[flip], rows[flip].copy()
    shuffled = QuboInstance("s", "s", base.n, base.diag, rows, cols, base.vals[order])
    p = lib.parameters(tolerance=1e-4 if use_float32 else 1e-7, use_float32=use_float32)
    out = {}
    for mode in ("direct", "staged"):
        monkeypatch.setenv("REFORM_PRAQ_UPLOAD", mode)
        out[mode] = [lib.solve(inst, p) for inst in (base, shuffled)]
        for k, (where, value) in enumerate(((base.edges - 1, base.n), (12345, None), (0, -1),
                                             (base.edges // 2, 1 << 32))):
            bad = QuboInstance("b", "b", base.n, base.diag, base.rows.copy(), base.cols.copy(), base.vals)
            if value is None:
                bad.cols[where] = bad.rows[where]    # a self-loop
            elif k % 2:
                bad.rows[where] = value
            else:
                bad.cols[where] = value
            assert lib.solve(bad, p).status == -2, (mode, where, value)
    for a, b in zip(out["direct"], out["staged"]):
        assert a.status == b.status == 0
        assert (a.iterations, a.lower, a.upper) == (b.iterations, b.lower, b.upper)
        assert np.array_equal(a.x, b.x)


@pytest.mark.parametrize("use_float32", [0, 1])
def test_slot1_layouts_agree(native, oracle_lib, monkeypatch, use_float32):
    """The two slot-1 layouts (push: scattered by the edge kernel; pull:
    gathered by the node kernel through the second-end index) add the same
    values in the same order, so a solve, its dual and a warm-started solve
    agree bit for bit; the pull layout also meets the max-flow roof dual.
    Unsorted, flipped edges exercise the warm start's edge permutation."""
    from reformulation_b200.praq import DeviceSolver, Library
    base = random_qubo(11, 500, 0.05)
    rng = np.random.default_rng(5)
    order = rng.permutation(base.edges)
    flip = rng.random(base.edges) < 0.5
    rows, cols = base.rows[order].copy(), base.cols[order].copy()
    rows[flip], cols[flip] = cols[flip], rows[flip].copy()
    inst = QuboInstance("s", "s", base.n, base.diag, rows, cols, base.vals[order])
    tol = 1e-4 if use_float32 else 1e-9
    p = Library().parameters(tolerance=tol, use_float32=use_float32)
    out = {}
    for layout in ("push", "pull"):
        monkeypatch.setenv("REFORM_PRAQ_SLOT1", layout)
        with DeviceSolver(inst, p) as dev:
            assert dev.run() == 0
            res, y = dev.result(want_x=True, want_dual=True)
            dev.set_warm(0.5 * (res.x + 0.5), y)
            assert dev.run() == 0
            warm = dev.result(want_x=True)
        out[layout] = (res, y, warm)
    (a, ya, wa), (b, yb, wb) = out["push"], out["pull"]
    assert (a.iterations, a.lower, a.upper) == (b.iterations, b.lower, b.upper)
    assert np.array_equal(a.x, b.x) and np.array_equal(ya, yb)
    assert (wa.iterations, wa.lower, wa.upper) == (wb.iterations, wb.lower, wb.upper)
    assert np.array_equal(wa.x, wb.x)
    if not use_float32:
        assert rel(b.upper, oracle_lib.roof_dual_maxflow(base)) <= 1e-7


@pytest.mark.parametrize("use_float32", [0, 1])
def test_slot1_layouts_agree_sequential_gather(native, monkeypatch, use_float32):
    """The same agreement with the node grid past one wave (n = 150,000), where
    the solver takes the sequential node gather: both layouts, bit for bit."""
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.praq import DeviceSolver, Library
    inst = qubo_uniform_edges(3, 150_000, 300_000)
    p = Library().parameters(tolerance=1e-4, use_float32=use_float32, max_iter=200)
    out = {}
    for layout in ("push", "pull"):
        monkeypatch.setenv("REFORM_PRAQ_SLOT1", layout)
        with DeviceSolver(inst, p) as dev:
            dev.run()
            out[layout] = dev.result(want_x=True, want_dual=True)
    (a, ya), (b, yb) = out["push"], out["pull"]
    assert (a.status, a.iterations, a.lower, a.upper) == (b.status, b.iterations, b.lower, b.upper)
    assert np.array_equal(a.x, b.x) and np.array_equal(ya, yb)
    assert a.lower <= a.upper


@pytest.mark.parametrize("seed,n,density", [(0, 8, 0.5), (1, 10, 0.4), (2, 12, 0.3), (3, 12, 0.6)])
def test_persistency_against_brute_force(lib, oracle_lib, seed, n, density):
    """Weak persistency of the roof dual (qubo/praq-jax/tests/test_solver.py):
    some binary minimiser of the QUBO, found by enumerating all 2^n points,
    takes every value the relaxation optimum fixes."""
    from reformulation_b200 import praq
    inst = random_qubo(100 + seed, n, density)
    s = lib.solve(inst, lib.parameters(tolerance=1e-10))
    assert s.status == 0
    fixed, vals = praq.persistent_variables(s.x)
    points = ((np.arange(1 << n)[:, None] >> np.arange(n)) & 1).astype(np.float64)
    values = np.array([oracle_lib.relaxation_value(inst, p) for p in points])
    best = values.min()
    assert s.lower <= best + 1e-9 * (1 + abs(best))     # the relaxation bounds the QUBO
    optima = points[values <= best + 1e-9 * (1 + abs(best))]
    assert np.any(np.all(optima[:, fixed] == vals[fixed], axis=1))


def test_time_limit_stops_with_a_valid_bracket(native, oracle_lib):
    """reform_praq_set_time_limit: a run past its budget stops between checks
    with PRAQ_STATUS_TIME_LIMIT and the bracket of the last completed check
    (both iterates are feasible, so it brackets the optimum); the backend
    reports status "time_limit" with those bounds."""
    from reformulation_b200 import praq
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.results import Tolerances
    inst = qubo_uniform_edges(6, 20_000, 100_000)
    flow = oracle_lib.roof_dual_maxflow(inst)
    p = praq.Library().parameters(tolerance=1e-12)
    with praq.DeviceSolver(inst, p) as dev:
        dev.set_time_limit(0.0)
        assert dev.run() == 2
        r = dev.result()
        assert r.status == 2 and 0 < r.iterations <= 64
        assert r.lower <= flow + 1e-9 * (1 + abs(flow)) <= r.upper + 2e-9 * (1 + abs(flow))
    res = praq.solve(inst, tolerances=Tolerances(optimality=1e-12), time_limit=0.0)
    assert res.status == "time_limit" and res.lower <= res.upper and np.isnan(res.objective)


def test_beyond_two_to_the_26_nodes(native, oracle_lib):
    """praq_solve takes the reference's sizes, n up to INT_MAX
    (qubo/praq-cuda/src/solver.cuh:525-526): n = 70,000,000 nodes (above
    2^26) and 300,000 uniform edges.  The optimum is the max-flow roof dual of
    the nodes the edges touch plus sum min(d_i, 0) over the others (an
    isolated node takes x_i = 1 exactly when d_i < 0)."""
    from reformulation_b200.instances import qubo_uniform_edges
    inst = qubo_uniform_edges(9, 70_000_000, 300_000)
    touched = np.unique(np.concatenate([inst.rows, inst.cols]))
    alone = np.ones(inst.n, bool)
    alone[touched] = False
    remap = np.full(inst.n, -1, np.int64)
    remap[touched] = np.arange(touched.size)
    sub = QuboInstance("sub", "sub", touched.size, inst.diag[touched], remap[inst.rows],
                       remap[inst.cols], inst.vals)
    opt = np.minimum(inst.diag[alone], 0.0).sum() + oracle_lib.roof_dual_maxflow(sub)
    from reformulation_b200.praq import Library
    lib = Library()
    s = lib.solve(inst, lib.parameters(tolerance=1e-7))
    assert s.status == 0 and s.gap <= 1e-7
    assert s.lower <= opt + 1e-9 * abs(opt) and s.upper >= opt - 1e-9 * abs(opt)
    assert rel(s.upper, opt) <= 1e-6
    assert np.all((s.x >= 0) & (s.x <= 1))


# ---- the persistent kernel for small instances ---------------------------------
# One cooperative launch per check block, the graph's tile functions in the
# graph's order with the graph's CTA shape: results equal the graph's bit for
# bit, and two runs equal each other (a grid-barrier race would break that),
# as the reference checks its PRIA megakernel (jrp/pria-cuda/tests/
# test_solver.cu:234-278).

def _praq_runs(inst, p, mode, runs=1, warm=None):
    from reformulation_b200.praq import DeviceSolver
    out = []
    with DeviceSolver(inst, p) as dev:
        active = dev.set_megakernel(mode)
        for _ in range(runs):
            assert dev.run() == 0
            out.append(dev.result(want_x=True, want_dual=True))
        if warm is not None:
            dev.set_warm(*warm)
            assert dev.run() == 0
            out.append(dev.result(want_x=True, want_dual=True))
        launches = dev.launches()
    return active, out, launches


@pytest.mark.parametrize("form", [1, 2], ids=["single-cta-or-grid", "grid"])
@pytest.mark.parametrize("use_float32", [0, 1])
@pytest.mark.parametrize("shape", ["n200", "n700", "n3000", "n12000"])
def test_persistent_kernel_equals_graph(native, use_float32, shape, form):
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.praq import Library
    inst = {"n200": lambda: qubo_sparse_bernoulli(0, 200, 0.05),
            "n700": lambda: qubo_uniform_edges(3, 700, 2000),
            "n3000": lambda: qubo_uniform_edges(2, 3000, 24000),
            "n12000": lambda: qubo_uniform_edges(4, 12000, 150000)}[shape]()
    p = Library().parameters(tolerance=1e-4 if use_float32 else 1e-7, use_float32=use_float32,
                             max_iter=100_000)
    rng = np.random.default_rng(1)
    warm = (rng.uniform(0, 1, inst.n), rng.normal(0, 5, (inst.edges, 2)))
    on, mega, ml = _praq_runs(inst, p, form, runs=2, warm=warm)
    off, graph, gl = _praq_runs(inst, p, 0, runs=1, warm=warm)
    assert off == 0
    assert on == (2 if form == 1 and shape in ("n200", "n700") else 1)
    for (a, ya), (b, yb) in ((mega[0], mega[1]), (mega[0], graph[0]), (mega[2], graph[1])):
        assert (a.iterations, a.lower, a.upper) == (b.iterations, b.lower, b.upper)
        assert np.array_equal(a.x, b.x) and np.array_equal(ya, yb)
    assert ml < gl


def test_persistent_kernel_choice_and_edgeless(native):
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.praq import DeviceSolver, Library
    p = Library().parameters(tolerance=1e-6)
    with DeviceSolver(qubo_sparse_bernoulli(0, 200, 0.05), p) as dev:
        assert dev.set_megakernel(-1) == 2             # fits one CTA: the single-CTA form
    with DeviceSolver(qubo_uniform_edges(2, 3000, 24000), p) as dev:
        assert dev.set_megakernel(-1) == 0             # does not fit: the graph
        assert dev.set_megakernel(1) == 1              # forced: the grid form
    inst = QuboInstance("e", "e", 5, np.array([-2.0, 1.0, 3.0, -1.0, 0.0]), np.zeros(0, np.int64),
                        np.zeros(0, np.int64), np.zeros(0))
    for form in (1, 2):
        with DeviceSolver(inst, Library().parameters(tolerance=1e-9, max_iter=10_000)) as dev:
            assert dev.set_megakernel(form) == 3 - form
            for _ in range(2):
                assert dev.run() == 0
                assert abs(dev.result().upper - (-3.0)) <= 1e-8


@pytest.mark.parametrize("case", ["grid", "single-cta"])
def test_persistent_kernel_time_limit(native, case):
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.praq import DeviceSolver, Library
    inst = qubo_uniform_edges(5, 3000, 24000) if case == "grid" else qubo_sparse_bernoulli(3, 300, 0.05)
    with DeviceSolver(inst, Library().parameters(tolerance=1e-15, max_iter=-1)) as dev:
        assert dev.set_megakernel(1) == (1 if case == "grid" else 2)
        dev.set_time_limit(0.0)
        assert dev.run() == 2                          # PRAQ_STATUS_TIME_LIMIT
        r = dev.result()
        assert r.lower <= r.upper and r.iterations > 0


def test_persistent_kernel_barrier_wait_runs_out(native):
    """Every barrier of the persistent kernel also waits for one CTA that is
    never launched (REFORM_PRAQ_MEGA_PHANTOM=1, a 50 ms wait limit): the first
    wait runs out, the kernel ends, the run returns PRAQ_ERROR_CUDA, and the
    same process then solves on the graph with the result of a clean
    process."""
    import os
    import subprocess
    import sys
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.praq import Library
    code = (
        "from reformulation_b200.praq import DeviceSolver, Library\n"
        "from reformulation_b200.instances import qubo_uniform_edges\n"
        "inst = qubo_uniform_edges(2, 3000, 24000)\n"
        "p = Library().parameters(tolerance=1e-6)\n"
        "with DeviceSolver(inst, p) as dev:\n"
        "    assert dev.set_megakernel(1)\n"
        "    st = dev.run()\n"
        "    assert st == -3, st\n"
        "    assert not dev.set_megakernel(0)\n"
        "    assert dev.run() == 0\n"
        "    a = dev.result()\n"
        "print(a.iterations, repr(a.upper), repr(a.lower))\n")
    env = dict(os.environ, REFORM_PRAQ_MEGA_PHANTOM="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    it, up, lo = out.stdout.split()[-3:]
    lib = Library()
    ref = lib.solve(qubo_uniform_edges(2, 3000, 24000), lib.parameters(tolerance=1e-6))
    assert int(it) == ref.iterations and float(up) == ref.upper and float(lo) == ref.lower


def test_convergence_trace(native):
    """The convergence trace (reform_praq_set_trace): one record per check,
    the start check first, then every op_steps block; the last record is the
    run's final check (its gap and bounds are the result's), restarts change
    omega only where the record says one was taken, and the records are the
    same in every form (graph, grid form, single CTA) and on a second run."""
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.praq import DeviceSolver, Library
    for inst in (qubo_sparse_bernoulli(0, 200, 0.05), qubo_uniform_edges(2, 3000, 24000)):
        p = Library().parameters(tolerance=1e-7, max_iter=100_000)
        traces = []
        for mode in (0, 1, 2):
            with DeviceSolver(inst, p) as dev:
                dev.set_megakernel(mode)
                dev.set_trace(4096)
                for _ in range(2):
                    assert dev.run() == 0
                    r = dev.result(want_x=False)
                    tr = dev.trace()
                    traces.append(tr)
        tr = traces[0]
        op = int(p.op_steps) if p.op_steps > 0 else int(tr["iteration"][1] - tr["iteration"][0])
        assert tr["restart"][0] == -1 and tr["iteration"][0] == 0
        assert np.all(np.diff(tr["iteration"]) == op)
        assert tr["terminated"][-1] == 1 and not tr["terminated"][:-1].any()
        assert tr["iteration"][-1] == r.iterations
        assert tr["gap"][-1] <= 1e-7 and (tr["gap"][:-1] > 1e-7).all()
        assert tr["lower"][-1] == r.lower and tr["upper"][-1] == r.upper
        taken = tr["restart"][1:-1] > 0
        changed = tr["omega"][1:] != tr["omega"][:-1]
        assert not (changed[:-1] & ~taken).any()          # omega moves only on a restart
        for other in traces[1:]:
            assert other.tobytes() == tr.tobytes()


def test_convergence_trace_ring_wraps(native):
    from reformulation_b200.praq import DeviceSolver, Library
    inst = qubo_sparse_bernoulli(0, 200, 0.05)
    with DeviceSolver(inst, Library().parameters(tolerance=1e-7, max_iter=100_000)) as dev:
        dev.set_trace(4096)
        assert len(dev.trace()) == 0                     # no run yet
        dev.run()
        full = dev.trace()
        dev.set_trace(3)
        dev.run()
        last = dev.trace()
        dev.set_trace(0)
        dev.run()
        assert len(dev.trace()) == 0
    assert len(full) > 3 and last.tobytes() == full[-3:].tobytes()
