"""The checked build (RB200_DEBUG_BOUNDS, `python -m reformulation_b200.build
--debug-bounds`): every gather and scatter index that comes from data is
range-checked on the device, a bad one is skipped and reported through the
run's status.  Small cases of every path run in a child process that loads the
checked library (REFORM_B200_LIB); each reports no caught index and gives the
release build's results -- PRAQ bit for bit (its step arithmetic has pinned
rounding, so the checks move nothing), PRIA within 1e-12 relative -- and the
release results themselves agree with the CPU oracle in the other suites.
This stands in for compute-sanitizer's memcheck, which this GPU pool does not
offer."""

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
DEBUG_LIB = ROOT / "reformulation_b200" / "_lib" / "libreform_b200_debug_bounds.so"

CHILD = r'''
import json, os, sys
sys.path.insert(0, os.environ["REPO_ROOT"])
from reformulation_b200 import praq, pria
from reformulation_b200.batch import Batch
from reformulation_b200.instances import jrp_demand, qubo_sparse_bernoulli, qubo_uniform_edges
out = {}
ql, jl = praq.Library(), pria.Library()
for name, inst in (("n200", qubo_sparse_bernoulli(0, 200, 0.05)), ("n3000", qubo_uniform_edges(2, 3000, 24000))):
    for f32 in (0, 1):
        for mode in (0, 1, 2):
            p = ql.parameters(tolerance=1e-6, use_float32=f32, max_iter=20000)
            with praq.DeviceSolver(inst, p) as dev:
                dev.set_megakernel(mode)
                st = dev.run()
                r = dev.result(want_x=False)
            out[f"praq-{name}-{f32}-{mode}"] = [st, r.iterations, r.lower, r.upper]
os.environ["REFORM_PRAQ_SLOT1"] = "pull"
inst = qubo_uniform_edges(2, 3000, 24000)
with praq.DeviceSolver(inst, ql.parameters(tolerance=1e-6, max_iter=20000)) as dev:
    st = dev.run()
    r = dev.result(want_x=False)
out["praq-pull"] = [st, r.iterations, r.lower, r.upper]
del os.environ["REFORM_PRAQ_SLOT1"]
for (n, t) in ((10, 25), (30, 75)):
    for prec in ("fp64", "mixed"):
        for mode in (0, 1):
            for extra in ({}, {"warm_steps": 2}):
                with pria.DeviceSolver(jrp_demand(9, n, t), jl.parameters(20000, 1e-6, **extra), prec) as dev:
                    dev.set_megakernel(mode)
                    st = dev.run()
                    r = dev.result()
                out[f"pria-{n}x{t}-{prec}-{mode}-{len(extra)}"] = [st, r.iterations, r.primal_objective, r.dual_objective]
with Batch("mixed") as b:
    ids = [b.add_qubo(q, ql.parameters(tolerance=1e-4, max_iter=20000))
           for q in (qubo_sparse_bernoulli(0, 200, 0.05), qubo_uniform_edges(2, 3000, 24000))]
    ids += [b.add_jrp(j, jl.parameters(20000, 1e-4)) for j in (jrp_demand(5, 10, 30), jrp_demand(7, 3, 17))]
    b.start()
    b.run()
    for k, i in enumerate(ids):
        r = b.result_qubo(i) if k < 2 else b.result_jrp(i)
        out[f"batch-{k}"] = [r.iterations, r.upper if k < 2 else r.primal_objective]
print(json.dumps(out))
'''


def _run(lib):
    env = dict(os.environ, REPO_ROOT=str(ROOT))
    env.pop("REFORM_B200_LIB", None)
    if lib:
        env["REFORM_B200_LIB"] = str(lib)
    res = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stderr[-3000:]
    return json.loads(res.stdout.strip().splitlines()[-1])


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def test_checked_build_catches_nothing_and_changes_nothing():
    if not DEBUG_LIB.exists():
        pytest.skip("the checked build is not built (python -m reformulation_b200.build --debug-bounds)")
    checked, release = _run(DEBUG_LIB), _run(None)
    assert checked.keys() == release.keys()
    for key, a in checked.items():
        b = release[key]
        if key.startswith("praq") or key.startswith("batch-0") or key.startswith("batch-1"):
            assert a == b, key                                   # status, iterations, bounds: bit for bit
        else:
            assert a[0] == b[0] and a[1] == b[1], key           # status (never REFORM_PRIA_STATUS_BOUNDS), iterations
            assert all(rel(x, y) <= 1e-12 for x, y in zip(a[2:], b[2:])), key
        if key.startswith("praq") or key.startswith("pria"):
            assert a[0] in (0, 1), key                           # 0 / 1: converged / not; never an error
