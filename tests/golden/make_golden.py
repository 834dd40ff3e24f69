"""Generate the golden fixtures from the REFERENCE itself (run once, in a
container that has the reference tree; the fixtures are committed, the GPU box
never reads the reference).

* praq_golden.json -- QUBO instances from the reference harness's own
  `random_instance` (qubo/harness/instances.py:264-283) and the BASELINE-style
  n=200 instance, each with the LP optimum from the reference's HiGHS wrapper
  (qubo/baselines/highs_backend.py) and our max-flow roof dual.
* pria_golden.json -- JRP instances from the reference harness's `random_jrp`
  (jrp/harness/instances.py:91-128) at the shapes of the reference's solver
  tests (jrp/pria-jax/tests/test_solver.py:34-43) and from ref::random_instance
  (jrp/pria-cuda/tests/ref_impl.hpp:56-80), each with the HiGHS optimum and the
  iterations / dual bound the reference's own CPU PRIA (ref::solve) reaches.

Usage: python tests/golden/make_golden.py [/path/to/reference]
"""

from __future__ import annotations

import importlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")


def _child(name: str):
    """Import the reference child project `name` ('qubo' or 'jrp') afresh."""
    for mod in [m for m in sys.modules if m.split(".")[0] in ("harness", "baselines")]:
        del sys.modules[mod]
    sys.path.insert(0, str(REF / name))
    try:
        instances = importlib.import_module("harness.instances")
        config = importlib.import_module("harness.config")
        highs = importlib.import_module("baselines.highs_backend")
    finally:
        sys.path.pop(0)
    return instances, config, highs


def praq_fixtures():
    sys.path.insert(0, str(ROOT))
    import oracle
    from reformulation_b200.instances import QuboInstance, qubo_sparse_bernoulli

    instances, config, highs = _child("qubo")
    out = []
    cases = [(0, 4, 1.0), (1, 6, 0.5), (2, 8, 0.2), (3, 8, 1.0), (4, 12, 0.5), (5, 20, 0.3),
             (6, 40, 0.2), (7, 60, 0.1)]
    for seed, n, density in cases:
        inst = instances.random_instance(seed, n, density)
        out.append((inst.name, inst))
    big = qubo_sparse_bernoulli(0, 200, 0.05)
    out.append((big.name, instances.Instance(big.name, "bernoulli", big.n, big.diag, big.rows,
                                             big.cols, big.vals)))
    records = []
    for name, inst in out:
        res = highs.solve(inst, tolerances=config.Tolerances(), time_limit=120.0)
        assert res.status == "optimal", (name, res)
        ours = QuboInstance(name, "golden", inst.n, np.asarray(inst.diag, float),
                            np.asarray(inst.rows, np.int64), np.asarray(inst.cols, np.int64),
                            np.asarray(inst.vals, float))
        records.append(dict(name=name, n=int(inst.n), diag=ours.diag.tolist(),
                            rows=ours.rows.tolist(), cols=ours.cols.tolist(),
                            vals=ours.vals.tolist(), highs=float(res.objective),
                            maxflow=float(oracle.roof_dual_maxflow(ours))))
    return dict(source="reference harness random_instance + HiGHS wrapper", instances=records)


def pria_fixtures():
    sys.path.insert(0, str(ROOT))
    import oracle
    from reformulation_b200.instances import JrpInstance

    instances, config, highs = _child("jrp")
    cases = []
    for seed, items, periods in ((1, 2, 3), (2, 3, 4), (3, 4, 7), (4, 5, 10), (5, 1, 6),
                                 (6, 1, 9)):
        inst = instances.random_jrp(seed, items, periods)
        cases.append((inst, 1e-6))
    for seed, n, t in ((101, 3, 7), (103, 10, 25)):
        r = oracle.ref_pria_random_instance(seed, n, t)
        cases.append((instances.Instance(r.name, "ref-random", r.order_costs, r.joint_order_cost,
                                         r.holding_costs), 1e-4))
    records = []
    for inst, tol in cases:
        res = highs.solve(inst, tolerances=config.Tolerances(), time_limit=120.0)
        assert res.status == "optimal", (inst.name, res)
        ours = JrpInstance(inst.name, "golden", np.asarray(inst.order_costs, float),
                           float(inst.joint_order_cost), np.asarray(inst.holding_costs, float))
        ref = oracle.ref_pria_solve(ours, oracle.pria_params(tolerance=tol))
        records.append(dict(name=inst.name, n=ours.items, t=ours.periods, k=ours.order_costs.tolist(),
                            k0=ours.joint_order_cost, h=ours.holding_costs.ravel().tolist(),
                            tol=tol, highs=float(res.objective),
                            ref_iterations=int(ref["iterations"]), ref_dual=float(ref["lower"]),
                            ref_primal=float(ref["upper"])))
    return dict(source="reference harness random_jrp / ref::random_instance + HiGHS + ref::solve",
                instances=records)


if __name__ == "__main__":
    (HERE / "praq_golden.json").write_text(json.dumps(praq_fixtures()))
    (HERE / "pria_golden.json").write_text(json.dumps(pria_fixtures()))
    print("wrote", HERE / "praq_golden.json", HERE / "pria_golden.json")
