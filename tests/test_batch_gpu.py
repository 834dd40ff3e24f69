"""The batched engine (include/reform.h) against solo solves: every instance
of a mixed QUBO + JRP batch of uneven sizes must reproduce its solo result
(reform_praq_* / reform_pria_*, same precision) BITWISE -- the engine runs the
same tile functions over the same per-instance layout -- including the
iteration count, which also shows per-instance restart and termination state
and retirement work.  Instances admitted while others run, removal, the
autotuner and the parity of a batch result with the oracle are checked too."""

import numpy as np
import pytest

from reformulation_b200.instances import jrp_demand, qubo_sparse_bernoulli, qubo_uniform_edges

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def mix():
    qs = [qubo_sparse_bernoulli(0, 200, 0.05), qubo_uniform_edges(2, 3000, 24000),
          qubo_uniform_edges(3, 700, 2000), qubo_uniform_edges(4, 12000, 150000)]
    js = [jrp_demand(5, 10, 30), jrp_demand(6, 40, 75), jrp_demand(7, 3, 17), jrp_demand(8, 60, 200)]
    return qs, js


def solo(qs, js, precision, tol):
    """Each instance alone.  A small JRP alone may run in the persistent
    kernel, whose FP32 z sums are taken over 256-thread CTAs (the batched
    engine's over 512, as the per-kernel graph's): FP32 solos take the graph,
    as the reference compares its batch with PRIA_MEGA=0 solos
    (jrp/pria-cuda/src/solver.cuh:635-641); FP64 solos keep the automatic
    choice, whose results are the graph's bit for bit."""
    from reformulation_b200 import praq, pria
    ql, jl = praq.Library(), pria.Library()
    out_q, out_j = [], []
    for q in qs:
        with praq.DeviceSolver(q, ql.parameters(tolerance=tol, max_iter=20000,
                                                use_float32=int(precision == "mixed"))) as d:
            assert d.run() == 0
            out_q.append(d.result())
    for j in js:
        with pria.DeviceSolver(j, jl.parameters(20000, tol), precision) as d:
            if precision == "mixed":
                d.set_megakernel(0)
            assert d.run() == 0
            out_j.append(d.result(want_solution=True))
    return out_q, out_j


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-4), ("fp64", 1e-6)])
def test_batch_equals_solo_bitwise(native, precision, tol):
    from reformulation_b200 import praq, pria
    from reformulation_b200.batch import Batch
    qs, js = mix()
    sq, sj = solo(qs, js, precision, tol)
    with Batch(precision) as b:
        qid = [b.add_qubo(q, praq.Library().parameters(tolerance=tol, max_iter=20000)) for q in qs]
        jid = [b.add_jrp(j, pria.Library().parameters(20000, tol)) for j in js]
        b.start()
        b.run()
        for i, q in enumerate(qs):
            r = b.result_qubo(qid[i])
            assert r.iterations == sq[i].iterations
            assert r.lower == sq[i].lower and r.upper == sq[i].upper
            assert np.array_equal(r.x, sq[i].x)
        for i, j in enumerate(js):
            r = b.result_jrp(jid[i], want_solution=True)
            assert r.iterations == sj[i].iterations
            assert r.primal_objective == sj[i].primal_objective
            assert r.dual_objective == sj[i].dual_objective
            assert np.array_equal(r.x, sj[i].x) and np.array_equal(r.z, sj[i].z)
        assert b.launches() > 0


def qp(tol=1e-4):
    from reformulation_b200 import praq
    return praq.Library().parameters(tolerance=tol, max_iter=20000)


def jp(tol=1e-4):
    from reformulation_b200 import pria
    return pria.Library().parameters(20000, tol)


def test_batch_admission_while_running_and_removal(native, oracle_lib):
    from reformulation_b200.batch import Batch
    qs, js = mix()
    sq, sj = solo(qs, js, "mixed", 1e-4)
    with Batch("mixed") as b:
        first = [b.add_qubo(qs[0], qp()), b.add_jrp(js[1], jp())]
        b.start()
        b.launch()
        b.launch()
        active, done = b.sync()
        finished = set(done)
        # two more join between blocks while the first ones run
        later = [b.add_qubo(qs[2], qp()), b.add_jrp(js[0], jp())]
        b.start()
        for _ in range(10000):
            while b.inflight() < 2:
                b.launch()
            active, done = b.sync()
            finished.update(done)
            if active == 0:
                break
        while b.inflight():
            b.sync()
        assert all(b.status(i)[0] for i in first + later)
        r = b.result_qubo(later[0])
        assert r.iterations == sq[2].iterations and np.array_equal(r.x, sq[2].x)
        rj = b.result_jrp(later[1])
        assert rj.iterations == sj[0].iterations and rj.primal_objective == sj[0].primal_objective
        before = b.device_bytes()
        b.remove(first[1])
        assert b.device_bytes() < before
        flow = oracle_lib.roof_dual_maxflow(qs[0])
        r0 = b.result_qubo(first[0])
        assert r0.lower <= flow + 1e-7 * (1 + abs(flow)) <= r0.upper + 2e-7 * (1 + abs(flow))
        assert r0.gap <= 1e-4


def test_autotune_keeps_results(native):
    from reformulation_b200 import praq
    from reformulation_b200.batch import Batch
    qs, js = mix()
    sq, sj = solo(qs[:2], js[:2], "mixed", 1e-4)
    with Batch("mixed") as b:
        ids = [b.add_qubo(q, qp()) for q in qs[:2]] + [b.add_jrp(j, jp()) for j in js[:2]]
        del ids
        b.start()
        shapes = b.autotune()
        assert shapes["grid_multiplier"] in (2, 4, 8, 16)
        b.run()
        for i in range(2):
            r = b.result_qubo(i)
            assert rel(r.upper, sq[i].upper) <= 1e-6 and r.status == 0
        for i in range(2):
            r = b.result_jrp(2 + i)
            assert r.iterations == sj[i].iterations


def test_long_horizon_added_before_short_ones(native):
    """Instances added largest first: the per-tile shared memory of a long
    horizon (T = 600, above the 48 KB default) must stay available after
    shorter instances join; each result still equals its solo run."""
    from reformulation_b200.batch import Batch
    js = [jrp_demand(30, 8, 600), jrp_demand(31, 3, 17), jrp_demand(32, 5, 40)]
    sq, sj = solo([], js, "mixed", 1e-4)
    with Batch("mixed") as b:
        ids = [b.add_jrp(j, jp()) for j in js]
        b.start()
        b.run()
        for i, j in zip(ids, sj):
            r = b.result_jrp(i)
            assert r.iterations == j.iterations and r.primal_objective == j.primal_objective


def test_warm_start_and_point_in_batch(native):
    """A warm-started QUBO in the batch equals the same warm start solo
    (bitwise); the point of a running instance can be read and the instance
    removed while others continue."""
    from reformulation_b200 import praq
    from reformulation_b200.batch import Batch
    qs, js = mix()
    lib = praq.Library()
    p = lib.parameters(tolerance=1e-6, max_iter=20000)
    rng = np.random.default_rng(9)
    warm = (rng.uniform(0, 1, qs[1].n), rng.normal(0, 20, (qs[1].edges, 2)))
    with praq.DeviceSolver(qs[1], p) as dev:
        dev.set_warm(*warm)
        assert dev.run() == 0
        solo = dev.result()
    with Batch("fp64") as b:
        a = b.add_qubo(qs[1], p)
        c = b.add_qubo(qs[3], p)
        b.set_warm_qubo(a, *warm)
        b.start()
        b.launch()
        b.sync()
        x, y = b.point_qubo(c)
        assert x.shape == (qs[3].n,) and y.shape == (qs[3].edges, 2)
        assert np.all((x >= 0) & (x <= 1))
        b.remove(c)                      # running: leaves the schedule
        b.run()
        r = b.result_qubo(a)
        assert r.iterations == solo.iterations and r.upper == solo.upper and r.lower == solo.lower


def test_escalation_continues_stalled_qubos_in_fp64(native, oracle_lib):
    """FP32 iterates cannot reach a 1e-8 gap; the escalating batch moves such a
    QUBO to FP64 at its last point and finishes it there, to the oracle's
    optimum.  A JRP in the same batch stays in FP32."""
    from reformulation_b200.batch import EscalatingBatch
    qs, js = mix()
    with EscalatingBatch(stall_iterations=256) as b:
        i = b.add_qubo(qs[2], qp(1e-8))
        k = b.add_jrp(js[0], jp(1e-4))
        b.start()
        b.run()
        assert i in b.escalated and k not in b.escalated
        r = b.result_qubo(i)
        assert r.status == 0 and (r.upper - r.lower) / (1 + abs(r.upper) + abs(r.lower)) <= 1e-8
        flow = oracle_lib.roof_dual_maxflow(qs[2])
        assert rel(r.upper, flow) <= 1e-7
        assert b.status(k)[0] and b.result_jrp(k).relative_gap <= 1e-4
