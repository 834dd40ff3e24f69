"""PRIA on the GPU against the oracles, through the C ABI.

Patterned on the reference's checks (jrp/pria-cuda/tests/test_solver.cu:37-389,
jrp/pria-jax/tests/test_solver.py:51-187): agreement with the reference's own
CPU solver ref::solve (iterations within one check interval, bounds), the HiGHS
optimum of the golden fixtures, a certificate recomputed on the host (primal
objective of the returned x, dual bound of the returned normalised y and z,
feasibility of all three), FP32 accuracy, the warm-start fixed point (even T:
zero iterations), odd-T padding, batch = solo, bad inputs, determinism.

Tolerances: FP64 bounds within 1e-6 relative of ref::solve's at the same
tolerance (different summation order: sort-based vs Michelot thresholds can
move a check by one block, so iterations within +-op_steps); objective within
10 x the solve tolerance of HiGHS; FP32 iterates within 1e-6 relative of FP64
at the same tolerance.
"""

import json
from pathlib import Path

import numpy as np
import pytest

from reformulation_b200.instances import JrpInstance, jrp_demand

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def jrp_from(rec):
    n, t = rec["n"], rec["t"]
    return JrpInstance(rec["name"], "golden", np.array(rec["k"], float), rec["k0"],
                       np.array(rec["h"], float).reshape(n, t, t))


@pytest.fixture(scope="module")
def lib(native):
    from reformulation_b200.pria import Library
    return Library()


def feasible(inst, s, tol=1e-9):
    x, y, z = s.x, s.y, s.z
    n, t = inst.items, inst.periods
    upper = np.triu(np.ones((t, t), bool))
    assert np.all(x >= -tol) and np.all(y >= -tol) and np.all(z >= -tol)
    assert np.all(x[:, ~upper] == 0) and np.all(y[:, ~upper] == 0)
    assert np.allclose(x.sum(axis=1), 1.0, atol=1e-7)          # sum_{s<=t} x = 1
    ok = inst.order_costs > 0
    # normalised duals: rows of y and groups of z sum to 1 on the padded
    # problem; an odd T drops the pad period from the output, so there they
    # sum to at most 1 (the dropped mass is nonnegative)
    ysum, zsum = y[ok].sum(axis=2), z.sum(axis=(0, 2))
    if t % 2 == 0:
        assert np.allclose(ysum, 1.0, atol=1e-7)
        if inst.joint_order_cost > 0:
            assert np.allclose(zsum, 1.0, atol=1e-7)
    else:
        assert np.all(ysum <= 1.0 + 1e-7) and np.all(zsum <= 1.0 + 1e-7)


@pytest.mark.parametrize("rec", json.loads((GOLDEN / "pria_golden.json").read_text())["instances"],
                         ids=lambda r: r["name"])
def test_golden_against_reference_and_highs(lib, oracle_lib, rec):
    inst = jrp_from(rec)
    s = lib.solve(inst, lib.parameters(-1, rec["tol"]), want_solution=True)
    assert s.status == 0
    assert abs(s.iterations - rec["ref_iterations"]) <= 16
    assert rel(s.dual_objective, rec["ref_dual"]) <= 1e-6
    assert rel(s.primal_objective, rec["highs"]) <= 10 * rec["tol"]
    assert s.dual_objective <= rec["highs"] + 1e-7 * (1 + abs(rec["highs"]))
    feasible(inst, s)
    assert rel(oracle_lib.pria_objective(inst, s.x), s.primal_objective) <= 1e-12
    assert oracle_lib.pria_dual_bound(inst, s.y, s.z) <= rec["highs"] + 1e-7 * (1 + abs(rec["highs"]))


@pytest.mark.parametrize("shape", [(3, 10, 25), (7, 8, 21), (9, 20, 50)])
def test_matches_reference_cpu_solver(lib, oracle_lib, shape):
    seed, n, t = shape
    inst = oracle_lib.ref_pria_random_instance(seed, n, t) if seed != 7 else jrp_demand(seed, n, t)
    p = oracle_lib.pria_params(tolerance=1e-6)
    ref = oracle_lib.ref_pria_solve(inst, p)
    s = lib.solve(inst, lib.parameters(-1, 1e-6), want_solution=True)
    assert s.status == 0 and s.relative_gap <= 1e-6
    assert abs(s.iterations - ref["iterations"]) <= 16
    assert rel(s.dual_objective, ref["lower"]) <= 1e-6
    assert rel(s.primal_objective, ref["upper"]) <= 1e-5
    feasible(inst, s)


def test_float32_accuracy(lib):
    """FP32 iterates: objective and dual bound within 1e-6 relative of the
    FP64 solve at the same 1e-4 gap tolerance."""
    inst = jrp_demand(11, 12, 40)
    a = lib.solve(inst, lib.parameters(-1, 1e-4))
    b = lib.solve(inst, lib.parameters(-1, 1e-4), precision="mixed", want_solution=True)
    assert b.status == 0 and b.relative_gap <= 1e-4
    assert rel(b.primal_objective, a.primal_objective) <= 1e-6
    assert rel(b.dual_objective, a.dual_objective) <= 1e-6
    assert b.x.dtype == np.float32


def test_warm_start_is_a_fixed_point(lib):
    inst = jrp_demand(12, 6, 20)             # even T: nothing padded
    s = lib.solve(inst, lib.parameters(-1, 1e-8), want_solution=True)
    w = lib.solve(inst, lib.parameters(-1, 1e-8), want_solution=True, warm=(s.x, s.y, s.z))
    assert w.status == 0
    assert w.iterations == 0
    assert rel(w.primal_objective, s.primal_objective) <= 1e-9


def test_odd_periods_are_padded(lib, oracle_lib):
    inst = jrp_demand(13, 5, 17)
    s = lib.solve(inst, lib.parameters(-1, 1e-7), want_solution=True)
    assert s.status == 0 and s.relative_gap <= 1e-7
    assert s.x.shape == (5, 17, 17)
    feasible(inst, s)
    ref = oracle_lib.pria_solve(inst, oracle_lib.pria_params(tolerance=1e-7))
    assert rel(s.primal_objective, ref["upper"]) <= 1e-6


def test_batch_equals_solo(native, lib):
    import ctypes

    from reformulation_b200 import _native
    insts = [jrp_demand(20 + b, 4, 12) for b in range(3)]
    n, t = 4, 12
    k = np.concatenate([i.order_costs for i in insts])
    k0 = np.array([i.joint_order_cost for i in insts])
    h = np.concatenate([i.holding_costs.ravel() for i in insts])
    x = np.empty(3 * n * t * t)
    infos = (_native.PriaResultInfo * 3)()
    p = lib.parameters(-1, 1e-7)
    st = _native.lib().pria_solve_batch_f64(3, n, t, _native.dptr(k), _native.dptr(k0), _native.dptr(h),
                                             ctypes.byref(p), _native.dptr(x), None, None, infos)
    assert st == 0
    for b, inst in enumerate(insts):
        s = lib.solve(inst, p, want_solution=True)
        assert infos[b].iterations == s.iterations
        assert infos[b].primal_objective == s.primal_objective
        assert np.array_equal(x[b * n * t * t:(b + 1) * n * t * t].reshape(n, t, t), s.x)


def test_rejects_bad_input(lib):
    inst = jrp_demand(1, 2, 4)
    bad = JrpInstance("b", "b", np.zeros(0), 1.0, np.zeros((0, 4, 4)))
    assert lib.solve(bad, lib.parameters()).status != 0
    big = JrpInstance("b", "b", np.ones(1), 1.0, np.zeros((1, 1030, 1030)))
    assert lib.solve(big, lib.parameters()).status != 0
    assert lib.solve(inst, lib.parameters()).status == 0


def test_max_iter_is_exact(lib):
    inst = jrp_demand(5, 10, 30)
    s = lib.solve(inst, lib.parameters(64, 1e-12))
    assert s.status == 0 and s.iterations == 64


def test_deterministic_and_backend(native):
    from reformulation_b200 import pria
    from reformulation_b200.results import Tolerances
    inst = jrp_demand(4, 15, 60)
    with pria.DeviceSolver(inst, pria.Library().parameters(-1, 1e-6)) as dev:
        dev.run()
        a = dev.result(want_solution=True)
        dev.run()
        b = dev.result(want_solution=True)
    assert a.iterations == b.iterations and a.primal_objective == b.primal_objective
    assert np.array_equal(a.x, b.x) and np.array_equal(a.z, b.z)
    r = pria.solve(inst, tolerances=Tolerances(optimality=1e-6), time_limit=60.0)
    assert r.status == "optimal" and r.objective == r.upper and r.entries == inst.entries
    m = pria.solve(inst, tolerances=Tolerances(optimality=1e-4), time_limit=60.0, precision="mixed")
    f = pria.solve(inst, tolerances=Tolerances(optimality=1e-4), time_limit=60.0)
    assert m.status == "optimal" and rel(m.objective, f.objective) <= 1e-6


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_solvers_of_different_sizes_coexist(native, precision):
    """A long horizon needs more dynamic shared memory per tile than the
    48 KB default; creating a smaller solver afterwards must not take that
    away from the larger one (the limit belongs to the kernel, not to a
    solver).  Both run, and the larger matches a solver created alone."""
    from reformulation_b200 import pria
    p = pria.Library().parameters(256, 1e-6)
    big, small = jrp_demand(30, 8, 600), jrp_demand(31, 3, 17)
    with pria.DeviceSolver(big, p, precision) as a, pria.DeviceSolver(small, p, precision) as b:
        assert a.run() == 0 and b.run() == 0
        ra = a.result()
    with pria.DeviceSolver(big, p, precision) as c:
        assert c.run() == 0
        rc = c.result()
    assert ra.iterations == rc.iterations and ra.primal_objective == rc.primal_objective


PLAIN_MODES = [dict(use_halpern=0, max_iter=96, tolerance=1e-12),
               dict(use_halpern=0, max_iter=-1, tolerance=1e-6),
               dict(warm_steps=3, tolerance=1e-6), dict(warm_steps=2, max_iter=16, tolerance=1e-12)]


@pytest.mark.parametrize("mode", PLAIN_MODES, ids=["vanilla-cap", "vanilla-tol", "warm3", "warm-past-cap"])
def test_vanilla_and_warm_phase_match_reference(lib, oracle_lib, mode):
    """Plain PDHG (use_halpern = 0, the CLI's `vanilla` flag) and warm_steps
    vanilla blocks before the Halpern method, against the reference's own CPU
    solver (jrp/pria-cuda/tests/ref_impl.hpp:297-330): the same iteration
    count (a cap is exact; the warm phase may run past max_iter, as the
    reference's does), bounds within 1e-6 relative."""
    inst = oracle_lib.ref_pria_random_instance(17, 5, 12)
    ref = oracle_lib.ref_pria_solve(inst, oracle_lib.pria_params(**mode))
    p = lib.parameters(mode.get("max_iter", -1), mode["tolerance"],
                       **{k: v for k, v in mode.items() if k not in ("max_iter", "tolerance")})
    s = lib.solve(inst, p, want_solution=True)
    assert s.status == 0
    if mode["tolerance"] < 1e-10:
        assert s.iterations == ref["iterations"]
    else:
        assert abs(s.iterations - ref["iterations"]) <= 16 and s.relative_gap <= mode["tolerance"]
    assert rel(s.dual_objective, ref["lower"]) <= 1e-6
    assert rel(s.primal_objective, ref["upper"]) <= 1e-6
    feasible(inst, s)
    # FP32 iterates: a 1e-4 gap, with a cap (they level off near 1e-6); the
    # objective within 1e-6 relative of the FP64 solve with the same parameters
    cap = mode.get("max_iter", -1)
    pm = lib.parameters(cap if cap > 0 else 5000, max(mode["tolerance"], 1e-4),
                        **{k: v for k, v in mode.items() if k not in ("max_iter", "tolerance")})
    m = lib.solve(inst, pm, precision="mixed")
    f = lib.solve(inst, pm)
    assert m.status == 0 and f.status == 0
    assert rel(m.primal_objective, f.primal_objective) <= 1e-6


def test_block_beyond_cluster_shared_memory(native):
    """A period block larger than a full cluster's shared-memory slices (FP64,
    N T above 196,608) takes the z half-step that recomputes z + r from global
    memory each Michelot round; it runs and agrees with the staged FP32 solve
    of the same instance to FP32 accuracy after the same iterations."""
    from reformulation_b200 import pria
    inst = jrp_demand(40, 400, 500)
    p = pria.Library().parameters(48, 1e-12)
    with pria.DeviceSolver(inst, p, "fp64") as a:
        assert a.run() == 0
        ra = a.result()
    with pria.DeviceSolver(inst, p, "mixed") as b:
        assert b.run() == 0
        rb = b.result()
    assert ra.iterations == rb.iterations == 48
    assert ra.dual_objective <= ra.primal_objective
    assert rel(ra.primal_objective, rb.primal_objective) <= 1e-3
    assert rel(ra.dual_objective, rb.dual_objective) <= 1e-3


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("shape", [(30, 400), (8, 300)])
def test_z_block_pairs_equal_single_blocks(native, monkeypatch, precision, shape):
    """The z half-step in pairs of period blocks (s, Tp - 1 - s) per cluster,
    the solver's choice in FP64 on large grids, adds every per-block sum in
    the order of one block per cluster: the same solve with either gives the
    same iterations, objectives and x, y, z bit for bit."""
    from reformulation_b200 import pria
    inst = jrp_demand(12, shape[0], shape[1])
    p = pria.Library().parameters(-1, 1e-6)
    out = {}
    for pair in ("0", "1"):
        monkeypatch.setenv("REFORM_PRIA_ZPAIR", pair)
        with pria.DeviceSolver(inst, p, precision) as dev:
            dev.set_megakernel(0)      # the graph's z kernel in both forms
            assert dev.run() == 0
            out[pair] = dev.result(want_solution=True)
    a, b = out["0"], out["1"]
    assert a.iterations == b.iterations
    assert a.primal_objective == b.primal_objective and a.dual_objective == b.dual_objective
    for k in ("x", "y", "z"):
        assert np.array_equal(getattr(a, k), getattr(b, k))


def test_concurrent_solves_from_host_threads(lib):
    """pria_solve is thread-safe (the reference's contract, pria.h): solves
    issued from several host threads at once, which share the library's
    pinned upload ring and device pool, equal the same solves run one after
    another, bit for bit."""
    from concurrent.futures import ThreadPoolExecutor
    insts = [jrp_demand(20 + k, 12 + 4 * k, 40 + 30 * k) for k in range(4)]
    p = lib.parameters(-1, 1e-6)
    alone = [lib.solve(j, p, precision=prec, want_solution=True)
             for j, prec in zip(insts, ["fp64", "mixed", "fp64", "mixed"])]
    with ThreadPoolExecutor(4) as ex:
        together = list(ex.map(lambda a: lib.solve(a[0], p, precision=a[1], want_solution=True),
                               zip(insts, ["fp64", "mixed", "fp64", "mixed"])))
    for a, b in zip(alone, together):
        assert a.iterations == b.iterations
        assert a.primal_objective == b.primal_objective and a.dual_objective == b.dual_objective
        assert np.array_equal(a.x, b.x) and np.array_equal(a.z, b.z)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zero_joint_and_item_costs_match_reference(lib, oracle_lib, precision):
    """The corners of the reference's checks (jrp/pria-jax/tests/test_solver.py):
    K0 = 0 (the z simplex is {0}: Michelot's threshold is +inf) and an item
    with K_i = 0 (its y rows are {0}); bounds agree with ref::solve and the
    returned point is feasible."""
    base = jrp_demand(31, 6, 20)
    k = base.order_costs.copy()
    k[2] = 0.0
    inst = JrpInstance("k0", "corner", k, 0.0, base.holding_costs)
    tol = 1e-6 if precision == "fp64" else 1e-4
    ref = oracle_lib.ref_pria_solve(inst, oracle_lib.pria_params(tolerance=tol))
    s = lib.solve(inst, lib.parameters(-1, tol), precision=precision, want_solution=True)
    assert s.status == 0 and s.relative_gap <= tol
    assert rel(s.dual_objective, ref["lower"]) <= 1e-6
    assert rel(s.primal_objective, ref["upper"]) <= (1e-5 if precision == "fp64" else 1e-6)
    assert np.all(s.z == 0) and np.all(s.y[2] == 0)
    if precision == "fp64":
        feasible(inst, s)


def test_time_limit_stops_with_a_valid_bracket(native, oracle_lib):
    """A wall-clock budget (reform_pria_set_time_limit) stops a long solve at a
    check and returns the bracket of that check; the backend reports status
    "time_limit" with those bounds (the reference's backend kills its solver
    past the limit, jrp/harness/backends/pria_cuda.py:114-145).  Without a
    budget the same solver runs on to the tolerance."""
    from reformulation_b200 import pria
    from reformulation_b200.results import Tolerances
    inst = jrp_demand(2, 60, 300)
    p = pria.Library().parameters(-1, 1e-12)
    with pria.DeviceSolver(inst, p, "mixed") as dev:
        dev.set_time_limit(0.0)
        assert dev.run() == pria.TIME_LIMIT
        r = dev.result(want_solution=True)
        assert 0 < r.iterations <= 64                       # stopped within two blocks
        assert r.dual_objective <= r.primal_objective
        assert rel(oracle_lib.pria_objective(inst, r.x), r.primal_objective) <= 1e-6
    res = pria.solve(inst, tolerances=Tolerances(optimality=1e-12), time_limit=0.0)
    assert res.status == "time_limit" and res.lower <= res.upper and np.isnan(res.objective)
    assert res.iterations > 0
    ok = pria.solve(jrp_demand(3, 8, 30), tolerances=Tolerances(optimality=1e-6), time_limit=60.0)
    assert ok.status == "optimal"


# ---- the persistent kernel for small instances ---------------------------------
# The reference's checks (jrp/pria-cuda/tests/test_solver.cu:234-278): two
# persistent-kernel runs are bitwise identical (a grid-barrier race would break
# that) and agree with the per-kernel path.  Here the FP64 persistent kernel
# runs the graph's tile functions in the graph's order with the same CTA
# shapes, so the agreement is bit for bit; FP32 z sums are taken over
# 256-thread CTAs (512 in the graph), so FP32 agrees within the objective
# tolerance.

def _mega_solve(inst, p, precision, mode, runs=1):
    from reformulation_b200 import pria
    out = []
    with pria.DeviceSolver(inst, p, precision) as dev:
        active = dev.set_megakernel(mode)
        for _ in range(runs):
            assert dev.run() == 0
            out.append(dev.result(want_solution=True))
        launches = dev.launches()
    return active, out, launches


def _same(a, b):
    assert a.iterations == b.iterations
    assert a.primal_objective == b.primal_objective and a.dual_objective == b.dual_objective
    for k in ("x", "y", "z"):
        assert np.array_equal(getattr(a, k), getattr(b, k))


@pytest.mark.parametrize("precision,items", [("fp64", 20), ("f32", 40)])
def test_large_solution_arrays_come_back_whole(lib, precision, items):
    """Solution arrays of 16 MB and more come back through the library's
    pinned ring, moved into the caller's arrays by several host threads: the
    objective of the returned x, recomputed on the host, is the one the
    device computed from its own copy, and x, y, z keep the solution's
    structure (17.4 MB an array here, in either precision)."""
    inst = jrp_demand(8, items, 330)
    s = lib.solve(inst, lib.parameters(-1, 1e-4), precision, want_solution=True)
    assert s.status == 0
    assert s.x.nbytes >= 16 << 20
    if precision == "fp64":
        feasible(inst, s)
    else:
        upper = np.triu(np.ones((330, 330), bool))
        assert np.all(s.x[:, ~upper] == 0) and np.all(s.y[:, ~upper] == 0)
        assert np.allclose(s.x.sum(axis=1, dtype=np.float64), 1.0, atol=1e-4)
    # the f32 solve holds H in FP32 (and takes it as FP32): its objective
    # is the host's to FP32 rounding of H; FP64 to summation order
    x = np.asarray(s.x, np.float64)
    assert rel(lib.objective(inst, x), s.primal_objective) <= (1e-6 if precision == "f32" else 1e-12)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gated_block_graph(native, precision):
    """A solver's first run launches its kernels one by one; later runs
    replay the captured check block, a conditional graph whose body runs only
    while the solve has not terminated.  The results are the first run's bit
    for bit, and a replayed run launches fewer kernels than the first (the
    block queued behind the one that ended the solve runs its gate alone)."""
    from reformulation_b200 import pria
    inst = jrp_demand(4, 40, 120)
    launches, out = [], []
    with pria.DeviceSolver(inst, pria.Library().parameters(-1, 1e-5), precision) as dev:
        dev.set_megakernel(0)
        for _ in range(3):
            assert dev.run() == 0
            out.append(dev.result(want_solution=True))
            launches.append(dev.launches())
    for b in out[1:]:
        _same(out[0], b)
    assert launches[1] < launches[0] and launches[2] == launches[1], launches


@pytest.mark.parametrize("shape", [(10, 25), (30, 75), (4, 12), (7, 9)])
def test_persistent_kernel_equals_graph_fp64(native, shape):
    from reformulation_b200 import pria
    inst = jrp_demand(40 + shape[0], *shape)
    p = pria.Library().parameters(-1, 1e-7)
    on, (m1, m2), mega_launches = _mega_solve(inst, p, "fp64", 1, runs=2)
    off, (g,), graph_launches = _mega_solve(inst, p, "fp64", 0)
    assert on and not off
    _same(m1, m2)                      # deterministic
    _same(m1, g)                       # the graph's result, bit for bit
    assert mega_launches < graph_launches
    assert m1.relative_gap <= 1e-7


@pytest.mark.parametrize("shape", [(10, 25), (30, 75)])
def test_persistent_kernel_fp32(native, shape):
    from reformulation_b200 import pria
    inst = jrp_demand(50 + shape[0], *shape)
    p = pria.Library().parameters(-1, 1e-4)
    on, (m1, m2), _ = _mega_solve(inst, p, "mixed", 1, runs=2)
    assert on
    _same(m1, m2)
    _, (g,), _ = _mega_solve(inst, p, "mixed", 0)
    _, (f,), _ = _mega_solve(inst, p, "fp64", 0)
    assert abs(m1.iterations - g.iterations) <= 2 * p.op_steps
    assert rel(m1.primal_objective, f.primal_objective) <= 1e-6
    assert rel(m1.primal_objective, g.primal_objective) <= 1e-6
    feasible(inst, m1, tol=1e-6)


@pytest.mark.parametrize("mode", PLAIN_MODES, ids=["vanilla-cap", "vanilla-tol", "warm3", "warm-past-cap"])
def test_persistent_kernel_vanilla_and_warm_phase(native, mode):
    """The vanilla blocks (plain PDHG, the warm phase) in the persistent kernel
    equal the graph's, FP64, bit for bit."""
    from reformulation_b200 import pria
    inst = jrp_demand(60, 5, 12)
    p = pria.Library().parameters(mode.get("max_iter", -1), mode["tolerance"],
                                  **{k: v for k, v in mode.items() if k not in ("max_iter", "tolerance")})
    on, (m,), _ = _mega_solve(inst, p, "fp64", 1)
    _, (g,), _ = _mega_solve(inst, p, "fp64", 0)
    assert on
    _same(m, g)


def test_persistent_kernel_choice(native):
    """Automatic: on for at most 16,384 packed entries, off above; forced on
    wherever one CTA holds every z period block, with the graph's result;
    never where it does not."""
    from reformulation_b200 import pria
    p = pria.Library().parameters(64, 1e-12)
    with pria.DeviceSolver(jrp_demand(70, 10, 25), p, "fp64") as dev:
        assert dev.set_megakernel(-1)
    big = jrp_demand(71, 60, 200)           # nd = 1.2M, one z block = 96,000 bytes in FP64
    with pria.DeviceSolver(big, p, "fp64") as dev:
        assert not dev.set_megakernel(-1)
    on, (m,), _ = _mega_solve(big, p, "fp64", 1)
    _, (g,), _ = _mega_solve(big, p, "fp64", 0)
    assert on and m.iterations == 64
    _same(m, g)
    with pria.DeviceSolver(jrp_demand(72, 300, 60), p, "fp64") as dev:   # z block 0: 144,000 bytes
        assert not dev.set_megakernel(1)


def test_persistent_kernel_time_limit_and_cap(native):
    from reformulation_b200 import pria
    inst = jrp_demand(73, 30, 75)
    _, (s,), _ = _mega_solve(inst, pria.Library().parameters(64, 1e-12), "fp64", 1)
    assert s.iterations == 64
    with pria.DeviceSolver(inst, pria.Library().parameters(-1, 1e-14), "fp64") as dev:
        assert dev.set_megakernel(1)
        dev.set_time_limit(0.0)
        assert dev.run() == pria.TIME_LIMIT
        r = dev.result()
        assert r.dual_objective <= r.primal_objective


def test_persistent_kernel_barrier_wait_runs_out(native):
    """Fault injection on the host side of the barrier: every barrier of the
    persistent kernel also waits for one CTA that is never launched
    (REFORM_PRIA_MEGA_PHANTOM=1, a 50 ms wait limit), so the first wait runs
    out; the kernel ends, the run returns cudaErrorLaunchTimeout (702), and
    the same process then solves on the graph and, with the injection off,
    with a new solver in the persistent kernel, with the results of a clean
    process."""
    import os
    import subprocess
    import sys
    from reformulation_b200 import pria
    code = (
        "from reformulation_b200 import pria\n"
        "from reformulation_b200.instances import jrp_demand\n"
        "inst = jrp_demand(74, 10, 25)\n"
        "p = pria.Library().parameters(-1, 1e-6)\n"
        "with pria.DeviceSolver(inst, p, 'fp64') as dev:\n"
        "    assert dev.set_megakernel(1)\n"
        "    st = dev.run()\n"
        "    assert st == 702, st\n"
        "    assert not dev.set_megakernel(0)\n"
        "    assert dev.run() == 0\n"
        "    a = dev.result()\n"
        "import os\n"
        "os.environ['REFORM_PRIA_MEGA_PHANTOM'] = '0'\n"
        "s = pria.Library().solve(inst, p)\n"
        "print(a.iterations, repr(a.primal_objective), s.iterations, repr(s.primal_objective))\n")
    env = dict(os.environ, REFORM_PRIA_MEGA_PHANTOM="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    it_a, obj_a, it_s, obj_s = out.stdout.split()[-4:]
    ref = pria.Library().solve(jrp_demand(74, 10, 25), pria.Library().parameters(-1, 1e-6))
    assert int(it_a) == int(it_s) == ref.iterations
    assert float(obj_a) == float(obj_s) == ref.primal_objective


@pytest.mark.parametrize("mode", [dict(), dict(warm_steps=2)], ids=["halpern", "warm-phase"])
def test_convergence_trace(native, mode):
    """The convergence trace (reform_pria_set_trace): the start check, the
    vanilla blocks and the end of the vanilla phase where there is one, then
    one record per op_steps block; the last is the final check (the result's
    gap and bounds); the same records on the graph and in the persistent
    kernel (FP64) and on a second run."""
    from reformulation_b200 import pria
    inst = jrp_demand(80, 10, 25)
    p = pria.Library().parameters(-1, 1e-7, **mode)
    traces = []
    for mega in (0, 1):
        with pria.DeviceSolver(inst, p, "fp64") as dev:
            dev.set_megakernel(mega)
            dev.set_trace(1024)
            for _ in range(2):
                assert dev.run() == 0
                r = dev.result()
                traces.append(dev.trace())
    tr = traces[0]
    assert tr["restart"][0] == -1
    if mode:
        assert list(tr["restart"][1:4]) == [4, 4, 5]
    assert tr["terminated"][-1] == 1 and not tr["terminated"][:-1].any()
    assert tr["iteration"][-1] == r.iterations and tr["gap"][-1] <= 1e-7
    assert np.all(np.diff(tr["iteration"]) >= 0) and (tr["gap"][:-1] > 1e-7).all()
    for other in traces[1:]:
        assert other.tobytes() == tr.tobytes()
