"""Parity at the benchmark workloads and at the stated tolerances, on the GPU.

Every solve is compared with a CPU oracle on the same seeded instance:

* the n = 100,000, m = 1,000,000 QUBO roof-dual LP (uniform distinct pairs,
  seed 1): FP64 on the GPU against the FP64 restatement (iterations within one
  check interval, bounds within 1e-8 relative) and against the reference's own
  praq-cuda built for sm_100a (the same iterations, bounds within 1e-12);
* FP32 iterates with FP64 reductions ("mixed") against the FP64 oracle at the
  same 1e-4 relative-gap tolerance: the objective (the upper bound the solve
  returns) within 1e-6 relative, the gap within 1e-4 -- for the n = 200 and
  n = 100,000 QUBOs, JRPs of 30 x 75 and 40 x 120 (the 100 x 500 workload's
  cost and demand distributions), and every instance of a batched mix;
* a JRP of 40 items and 120 periods, FP64, against the reference's own CPU
  solver ref::solve (jrp/pria-cuda/tests/ref_impl.hpp), as the reference's
  own certificate test does (jrp/pria-cuda/tests/test_solver.cu:324-386);
* every QUBO of the committed HiGHS fixtures (tests/golden/praq_golden.json,
  written by the reference's own HiGHS wrapper) against its HiGHS optimum and
  max-flow roof dual, as qubo/praq-cuda/tests/test_solver.cu:122-262 checks
  the enumerated optimum.

Tolerances are written where they are used: `OBJ_TOL` = 1e-6 relative
objective (|a - b| / (1 + |b|)), `GAP_TOL` = 1e-4 relative gap.
"""

import json
from pathlib import Path

import numpy as np
import pytest

from reformulation_b200.instances import (QuboInstance, jrp_demand, qubo_sparse_bernoulli,
                                          qubo_uniform_edges)

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
OBJ_TOL = 1e-6
GAP_TOL = 1e-4


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


@pytest.fixture(scope="module")
def cfg2():
    return qubo_uniform_edges(1, 100_000, 1_000_000)


@pytest.fixture(scope="module")
def cfg2_oracle(oracle_lib, cfg2):
    return oracle_lib.praq_solve(cfg2, oracle_lib.praq_params(tolerance=GAP_TOL),
                                 threads=oracle_lib.threads_available())


def gpu_praq(inst, tol, use_float32):
    from reformulation_b200.praq import Library
    lib = Library()
    return lib.solve(inst, lib.parameters(tolerance=tol, use_float32=use_float32))


def test_large_qubo_fp64_matches_oracle(native, cfg2, cfg2_oracle):
    ref = cfg2_oracle
    s = gpu_praq(cfg2, GAP_TOL, 0)
    assert s.status == 0 and ref["status"] == 0
    assert abs(s.iterations - ref["iterations"]) <= 16
    assert rel(s.upper, ref["upper"]) <= 1e-8
    assert rel(s.lower, ref["lower"]) <= 1e-8
    assert s.gap <= GAP_TOL


def test_large_qubo_fp64_matches_reference_praq_cuda(native, oracle_lib, cfg2):
    """The reference's praq-cuda, compiled in place for sm_100a, on the same
    GPU: the same iteration count and the same bounds to 1e-12."""
    from oracle import REF_PRAQ
    if not REF_PRAQ.exists():
        pytest.skip("the reference's praq-cuda was not built (no reference tree at build time)")
    ref = oracle_lib.RefPraq().solve(cfg2, tolerance=GAP_TOL)
    s = gpu_praq(cfg2, GAP_TOL, 0)
    assert ref["status"] == 0 and s.status == 0
    assert s.iterations == ref["iterations"]
    assert rel(s.upper, ref["upper"]) <= 1e-12
    assert rel(s.lower, ref["lower"]) <= 1e-12


def test_large_qubo_mixed_objective_within_tolerance(native, oracle_lib, cfg2, cfg2_oracle):
    s = gpu_praq(cfg2, GAP_TOL, 1)
    assert s.status == 0 and s.gap <= GAP_TOL
    assert rel(s.upper, cfg2_oracle["upper"]) <= OBJ_TOL
    flow = oracle_lib.roof_dual_maxflow(cfg2)
    assert s.lower <= flow + 1e-9 * (1 + abs(flow)) <= s.upper + 2e-9 * (1 + abs(flow))


def test_small_qubo_mixed_objective_within_tolerance(native, oracle_lib):
    inst = qubo_sparse_bernoulli(0, 200, 0.05)
    ref = oracle_lib.praq_solve(inst, oracle_lib.praq_params(tolerance=GAP_TOL))
    s = gpu_praq(inst, GAP_TOL, 1)
    assert s.status == 0 and s.gap <= GAP_TOL
    assert rel(s.upper, ref["upper"]) <= OBJ_TOL
    f64 = gpu_praq(inst, GAP_TOL, 0)
    assert rel(f64.upper, ref["upper"]) <= 1e-9 and f64.iterations == ref["iterations"]


@pytest.mark.parametrize("shape", [(6, 30, 75), (2, 40, 120)], ids=["30x75", "40x120"])
def test_jrp_mixed_objective_within_tolerance(native, oracle_lib, shape):
    from reformulation_b200.pria import Library
    seed, n, t = shape
    inst = jrp_demand(seed, n, t)
    ref = oracle_lib.ref_pria_solve(inst, oracle_lib.pria_params(tolerance=GAP_TOL))
    lib = Library()
    s = lib.solve(inst, lib.parameters(-1, GAP_TOL), precision="mixed")
    assert s.status == 0 and s.relative_gap <= GAP_TOL
    assert rel(s.primal_objective, ref["upper"]) <= OBJ_TOL
    assert rel(s.dual_objective, ref["lower"]) <= OBJ_TOL


def test_jrp_40x120_fp64_matches_reference_cpu_solver(native, oracle_lib):
    from reformulation_b200.pria import Library
    inst = jrp_demand(2, 40, 120)
    ref = oracle_lib.ref_pria_solve(inst, oracle_lib.pria_params(tolerance=GAP_TOL))
    lib = Library()
    s = lib.solve(inst, lib.parameters(-1, GAP_TOL), want_solution=True)
    assert s.status == 0 and s.relative_gap <= GAP_TOL
    assert abs(s.iterations - ref["iterations"]) <= 16
    assert rel(s.primal_objective, ref["upper"]) <= 1e-8
    assert rel(s.dual_objective, ref["lower"]) <= 1e-8
    assert rel(oracle_lib.pria_objective(inst, s.x), s.primal_objective) <= 1e-12
    assert oracle_lib.pria_dual_bound(inst, s.y, s.z) <= s.primal_objective


def test_batch_mix_each_result_within_tolerance(native, oracle_lib):
    """Every instance of an uneven QUBO + JRP batch, solved in the batched
    engine with FP32 iterates, against the FP64 oracle of that instance."""
    from reformulation_b200 import praq, pria
    from reformulation_b200.batch import Batch
    qs = [qubo_sparse_bernoulli(0, 200, 0.05), qubo_uniform_edges(2, 3000, 24000),
          qubo_uniform_edges(3, 700, 2000), qubo_uniform_edges(4, 12000, 150000)]
    js = [jrp_demand(5, 10, 30), jrp_demand(6, 40, 75), jrp_demand(7, 3, 17),
          jrp_demand(8, 60, 200)]
    threads = oracle_lib.threads_available()
    with Batch("mixed") as b:
        qid = [b.add_qubo(q, praq.Library().parameters(tolerance=GAP_TOL, max_iter=20000))
               for q in qs]
        jid = [b.add_jrp(j, pria.Library().parameters(20000, GAP_TOL)) for j in js]
        b.start()
        b.run()
        for i, q in zip(qid, qs):
            r = b.result_qubo(i)
            ref = oracle_lib.praq_solve(q, oracle_lib.praq_params(tolerance=GAP_TOL),
                                        threads=threads)
            assert r.status == 0 and r.gap <= GAP_TOL, q.name
            assert rel(r.upper, ref["upper"]) <= OBJ_TOL, (q.name, r.upper, ref["upper"])
        for i, j in zip(jid, js):
            r = b.result_jrp(i)
            ref = oracle_lib.pria_solve(j, oracle_lib.pria_params(tolerance=GAP_TOL),
                                        threads=threads)
            assert r.relative_gap <= GAP_TOL, j.name
            assert rel(r.primal_objective, ref["upper"]) <= OBJ_TOL, (j.name, r.primal_objective,
                                                                       ref["upper"])


def golden_qubos():
    return json.loads((GOLDEN / "praq_golden.json").read_text())["instances"]


@pytest.mark.parametrize("rec", golden_qubos(), ids=lambda r: r["name"])
def test_golden_qubos_against_highs(native, rec):
    inst = QuboInstance(rec["name"], "golden", rec["n"], np.array(rec["diag"], float),
                        np.array(rec["rows"], np.int64), np.array(rec["cols"], np.int64),
                        np.array(rec["vals"], float))
    s = gpu_praq(inst, 1e-9, 0)
    assert s.status == 0 and s.gap <= 1e-9
    assert rel(s.upper, rec["highs"]) <= OBJ_TOL
    assert rel(s.upper, rec["maxflow"]) <= OBJ_TOL
    assert s.lower <= rec["highs"] + 1e-6 * (1 + abs(rec["highs"]))
    m = gpu_praq(inst, GAP_TOL, 1)
    assert m.status == 0 and m.gap <= GAP_TOL
    assert m.lower <= rec["maxflow"] + 1e-7 * (1 + abs(rec["maxflow"])) <= m.upper + 2e-7 * (1 + abs(rec["maxflow"]))
