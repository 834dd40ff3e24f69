"""The oracles, pinned (CPU only): the PRAQ restatement against the enumerated
half-integral optimum, the max-flow roof dual and the committed HiGHS values of
tests/golden; the PRIA restatement against the reference's own ref_impl.hpp
(compiled in place into oracle/_ref) and against the committed HiGHS values."""

import json
from pathlib import Path

import numpy as np
import pytest

from reformulation_b200.instances import JrpInstance, QuboInstance

GOLDEN = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def load(name):
    return json.loads((GOLDEN / name).read_text())


def qubo_from(rec):
    return QuboInstance(rec["name"], "golden", rec["n"], np.array(rec["diag"], float),
                        np.array(rec["rows"], np.int64), np.array(rec["cols"], np.int64),
                        np.array(rec["vals"], float))


def jrp_from(rec):
    n, t = rec["n"], rec["t"]
    return JrpInstance(rec["name"], "golden", np.array(rec["k"], float), rec["k0"],
                       np.array(rec["h"], float).reshape(n, t, t))


def test_check_interval_values(oracle_lib):
    assert oracle_lib.check_interval(50_000) == 2
    assert oracle_lib.check_interval(400_000) == 9
    assert oracle_lib.check_interval(2_000_000) == 16
    assert oracle_lib.check_interval(int(50000.0 * 7.38905609893065), power=0.5) == 15


@pytest.mark.parametrize("rec", load("praq_golden.json")["instances"], ids=lambda r: r["name"])
def test_praq_oracle_against_highs_and_maxflow(oracle_lib, rec):
    inst = qubo_from(rec)
    r = oracle_lib.praq_solve(inst, oracle_lib.praq_params(tolerance=1e-9))
    assert r["status"] == 0
    assert rel(r["upper"], rec["highs"]) <= 1e-6
    assert rel(r["upper"], rec["maxflow"]) <= 1e-6
    assert r["lower"] <= rec["highs"] + 1e-6 * (1 + abs(rec["highs"]))
    if inst.n <= 8:
        assert rel(r["upper"], oracle_lib.half_integral_optimum(inst)) <= 1e-7
    assert rel(oracle_lib.relaxation_value(inst, r["x"]), r["upper"]) <= 1e-9


def test_praq_oracle_bounds_bracket_under_caps(oracle_lib):
    rec = load("praq_golden.json")["instances"][0]
    inst = qubo_from(rec)
    for cap in (1, 4, 16, 64):
        r = oracle_lib.praq_solve(inst, oracle_lib.praq_params(tolerance=1e-12, max_iter=cap))
        assert r["lower"] <= rec["highs"] + 1e-9 * (1 + abs(rec["highs"]))
        assert r["upper"] >= rec["highs"] - 1e-9 * (1 + abs(rec["highs"]))


@pytest.mark.parametrize("rec", load("pria_golden.json")["instances"], ids=lambda r: r["name"])
def test_pria_oracle_against_reference_and_highs(oracle_lib, rec):
    inst = jrp_from(rec)
    p = oracle_lib.pria_params(tolerance=rec["tol"])
    r = oracle_lib.pria_solve(inst, p, want_solution=True)
    # the reference's own CPU PRIA, as recorded when the fixture was made
    assert r["iterations"] == rec["ref_iterations"]
    assert rel(r["lower"], rec["ref_dual"]) <= 1e-9
    assert rel(r["upper"], rec["highs"]) <= 10 * rec["tol"]
    assert r["lower"] <= rec["highs"] + 1e-7 * (1 + abs(rec["highs"]))
    # host-recomputed certificate
    assert rel(oracle_lib.pria_objective(inst, r["x"]), r["upper"]) <= 1e-12
    assert oracle_lib.pria_dual_bound(inst, r["y"], r["z"]) <= rec["highs"] + 1e-7 * (1 + abs(rec["highs"]))


def test_pria_oracle_matches_reference_live(oracle_lib):
    if not oracle_lib.ref_pria_available():
        pytest.skip("oracle/_ref not built")
    inst = oracle_lib.ref_pria_random_instance(131, 6, 13)
    p = oracle_lib.pria_params(tolerance=1e-6)
    a = oracle_lib.pria_solve(inst, p)
    b = oracle_lib.ref_pria_solve(inst, p)
    assert a["iterations"] == b["iterations"]
    assert rel(a["lower"], b["lower"]) <= 1e-9


PRIA_PLAIN_MODES = [dict(use_halpern=0, max_iter=96, tolerance=1e-12),
                    dict(use_halpern=0, max_iter=-1, tolerance=1e-6),
                    dict(warm_steps=3, tolerance=1e-6), dict(warm_steps=2, max_iter=16, tolerance=1e-12)]
PRIA_PLAIN_IDS = ["vanilla-cap", "vanilla-tol", "warm3", "warm-past-cap"]


@pytest.mark.parametrize("mode", PRIA_PLAIN_MODES, ids=PRIA_PLAIN_IDS)
def test_pria_oracle_vanilla_and_warm_phase_match_reference(oracle_lib, mode):
    """Plain PDHG (use_halpern = 0) and the vanilla warm phase before Halpern
    (warm_steps > 0) of jrp/pria-cuda/tests/ref_impl.hpp:297-330."""
    if not oracle_lib.ref_pria_available():
        pytest.skip("oracle/_ref not built")
    inst = oracle_lib.ref_pria_random_instance(17, 5, 12)
    p = oracle_lib.pria_params(**mode)
    a = oracle_lib.pria_solve(inst, p)
    b = oracle_lib.ref_pria_solve(inst, p)
    assert a["iterations"] == b["iterations"]
    assert rel(a["lower"], b["lower"]) <= 1e-9 and rel(a["upper"], b["upper"]) <= 1e-9


def test_maxflow_matches_enumeration(oracle_lib):
    rng = np.random.default_rng(5)
    for k in range(20):
        n = int(rng.integers(2, 8))
        iu = np.triu_indices(n, 1)
        keep = rng.random(iu[0].size) < 0.6
        vals = rng.integers(-5, 6, keep.sum()).astype(float)
        inst = QuboInstance("m", "m", n, rng.integers(-5, 6, n).astype(float), iu[0][keep],
                            iu[1][keep], vals)
        assert abs(oracle_lib.roof_dual_maxflow(inst) - oracle_lib.half_integral_optimum(inst)) < 1e-9
