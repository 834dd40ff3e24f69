"""The continuous-batching request loop (reformulation_b200.serving): requests
arriving over time are admitted between block replays, run in the same graph
replays as the others, and retire as they converge.  Each result must be the
same served alone and served in the mix: bitwise (same engine, same kernels,
same per-instance layout), and within the stated tolerance of the plain
single-instance solvers (1e-6 relative objective at a 1e-4 gap; the
demand-form JRP builds its costs on the device, so its last bits may differ
from the dense input's)."""

import numpy as np
import pytest

from reformulation_b200.instances import JrpSpec, qubo_uniform_edges

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def requests():
    from reformulation_b200.serving import Request
    rng = np.random.default_rng(41)
    reqs = []
    for k in range(10):
        if k % 3 == 2:
            n, t = int(rng.integers(4, 20)), int(rng.integers(10, 60))
            d = rng.integers(1, 101, (n, t)).astype(float)
            d[rng.random((n, t)) < 0.3] = 0.0
            inst = JrpSpec(f"j{k}", rng.uniform(10, 50, n), float(rng.uniform(50, 150)),
                           rng.uniform(0.1, 1.0, n), d)
        else:
            n = int(rng.integers(200, 3000))
            inst = qubo_uniform_edges(100 + k, n, int(n * rng.uniform(2, 12)))
        reqs.append(Request(k, 0.02 * k, inst))
    return reqs


def test_serving_mix_equals_alone_and_solo(native):
    from reformulation_b200 import praq, pria
    from reformulation_b200.serving import Request, Server, percentiles
    reqs = requests()
    server = Server(budget_bytes=2e9, tolerance=1e-4)
    done = {c.rid: c for c in server.serve(reqs)}
    server.close()
    assert sorted(done) == list(range(len(reqs)))
    lat = [c.latency for c in done.values()]
    assert all(v >= 0 for v in lat) and np.isfinite(percentiles(lat)["p99"])
    for req in reqs:
        alone = Server(budget_bytes=2e9, tolerance=1e-4)
        a = alone.serve([Request(req.rid, 0.0, req.instance)])[0]
        alone.close()
        c = done[req.rid]
        assert (a.iterations, a.lower, a.upper) == (c.iterations, c.lower, c.upper)
        assert c.gap <= 1e-4
        if req.kind == "qubo":
            lib = praq.Library()
            s = lib.solve(req.instance, lib.parameters(tolerance=1e-4, use_float32=1))
            assert s.iterations == c.iterations and s.upper == c.upper
        else:
            lib = pria.Library()
            s = lib.solve(req.instance.build(), lib.parameters(-1, 1e-4), precision="mixed")
            assert rel(s.primal_objective, c.upper) <= 1e-6
            assert abs(s.iterations - c.iterations) <= 16


def test_budget_limits_admission(native):
    from reformulation_b200.serving import Server, footprint
    reqs = requests()[:6]
    small = max(footprint(r.instance) for r in reqs)
    server = Server(budget_bytes=1.5 * small, tolerance=1e-4)
    done = server.serve(reqs)
    server.close()
    assert len(done) == len(reqs)
    # never more than what one (or two small) instances need was held at once
    assert server.high_water <= 3 * small
