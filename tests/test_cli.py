"""The file CLIs praq_solve_file / pria_solve_file, which the reference's
harness backends drive as subprocesses (qubo/harness/backends/praq_cuda.py:27-86,
jrp/harness/backends/pria_cuda.py).  The instance/result wire formats, the
flags and the exit codes are the contract of qubo/praq-cuda/tools/
praq_solve_file.cu:7-31 and jrp/pria-cuda/tools/pria_solve_file.cu:7-45.

CPU tests: every exit-2 path (usage, unreadable or malformed input), which is
reached before any CUDA call; the shared wire-format module
(cli/wire_format.hpp) on its own, through tests/wire_format_check.cpp; and,
where the reference tree is present, the reference's own harness code against
this library: its backends' instance writers and result readers, its ctypes
wrappers loading libreform_b200.so, and its subprocess backend running the CLI.
GPU tests: a solve through the CLI equals the same solve through the C ABI bit
for bit (bounds, iterations, x), on files written by the test and on the
committed files written by the reference's harness (tests/golden/wire/); the
stdout "key: value" lines the harness parses, the solution flag and the f32
flag.
"""

import json
import os
import struct
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

from reformulation_b200.instances import QuboInstance, jrp_demand, qubo_sparse_bernoulli

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
GOLDEN = HERE / "golden" / "wire"

PRAQ_MAGIC, PRIA_MAGIC = 0x51415250, 0x41495250


@pytest.fixture(scope="module")
def bins(native):
    from reformulation_b200 import build
    exes = {exe.name: exe for exe in build.build_cli()}
    return exes["praq_solve_file"], exes["pria_solve_file"]


def write_praq(inst, path):
    with open(path, "wb") as f:
        f.write(np.array([PRAQ_MAGIC, inst.n, inst.edges], "<i8").tobytes())
        f.write(np.ascontiguousarray(inst.diag, "<f8").tobytes())
        f.write(np.ascontiguousarray(inst.rows, "<i8").tobytes())
        f.write(np.ascontiguousarray(inst.cols, "<i8").tobytes())
        f.write(np.ascontiguousarray(inst.vals, "<f8").tobytes())


def read_praq(path):
    data = path.read_bytes()
    n, iters, status = struct.unpack_from("<qqq", data, 0)
    lower, upper = struct.unpack_from("<dd", data, 24)
    return iters, status, lower, upper, np.frombuffer(data, "<f8", n, 40)


def write_pria(inst, path):
    with open(path, "wb") as f:
        f.write(np.array([PRIA_MAGIC, inst.items, inst.periods], "<i8").tobytes())
        f.write(np.array([inst.joint_order_cost], "<f8").tobytes())
        f.write(np.ascontiguousarray(inst.order_costs, "<f8").tobytes())
        f.write(np.ascontiguousarray(inst.holding_costs, "<f8").tobytes())


def read_pria(path, solution=False):
    data = path.read_bytes()
    n, t, iters, status = struct.unpack_from("<qqqq", data, 0)
    lower, upper, gap = struct.unpack_from("<ddd", data, 32)
    out = dict(n=n, t=t, iterations=iters, status=status, lower=lower, upper=upper, gap=gap)
    if solution:
        size = n * t * t
        arr = np.frombuffer(data, "<f8", 3 * size, 56).reshape(3, n, t, t)
        out.update(x=arr[0], y=arr[1], z=arr[2])
    else:
        assert len(data) == 56
    return out


def keys(stdout):
    out = {}
    for line in stdout.splitlines():
        k, sep, v = line.partition(":")
        if sep:
            out[k.strip()] = v.strip()
    return out


def run(*args):
    return subprocess.run([str(a) for a in args], capture_output=True, text=True, timeout=300)


# ---- CPU: the exit-2 contract -------------------------------------------------

def test_usage_and_unreadable_input(bins, tmp_path):
    praq, pria = bins
    assert run(praq).returncode == 2
    assert run(praq, "a").returncode == 2
    assert run(praq, "a", "b", "1e-4", "10", "f32", "extra").returncode == 2
    assert run(praq, "a", "b", "1e-4", "10", "solution").returncode == 2    # a PRIA-only flag
    assert run(pria).returncode == 2
    assert run(praq, tmp_path / "missing", tmp_path / "r").returncode == 2
    assert run(pria, tmp_path / "missing", tmp_path / "r").returncode == 2
    inst = tmp_path / "i"
    inst.write_bytes(b"")
    assert run(pria, inst, tmp_path / "r", "1e-4", "-1", "bogus").returncode == 2
    r = run(pria, inst, tmp_path / "r")
    assert r.returncode == 2 and r.stderr.startswith("pria_solve_file: ")
    assert not (tmp_path / "r").exists()


def test_malformed_files_are_rejected(bins, tmp_path):
    praq, pria = bins
    q = qubo_sparse_bernoulli(0, 20, 0.3)
    good = tmp_path / "q.bin"
    write_praq(q, good)
    raw = good.read_bytes()
    for name, data, why in (("magic", struct.pack("<q", 7) + raw[8:], "wrong magic"),
                            ("short", raw[:-8], "size mismatch"),
                            ("long", raw + b"\0" * 8, "size mismatch"),
                            ("negative", raw[:8] + struct.pack("<q", -1) + raw[16:], "bad header"),
                            ("huge", raw[:16] + struct.pack("<q", 1 << 61) + raw[24:], "size mismatch")):
        f = tmp_path / name
        f.write_bytes(data)
        r = run(praq, f, tmp_path / "r")
        assert r.returncode == 2 and why in r.stderr, (name, r.stderr)
        assert not (tmp_path / "r").exists()
    j = jrp_demand(1, 2, 4)
    pj = tmp_path / "j.bin"
    write_pria(j, pj)
    raw = pj.read_bytes()
    for name, data, why in (("jmagic", struct.pack("<q", PRAQ_MAGIC) + raw[8:], "wrong magic"),
                            ("jshort", raw[:-8], "size mismatch"),
                            ("jzero", raw[:8] + struct.pack("<q", 0) + raw[16:], "bad header"),
                            ("jhuge", raw[:16] + struct.pack("<q", 1 << 31) + raw[24:], "size mismatch")):
        f = tmp_path / name
        f.write_bytes(data)
        r = run(pria, f, tmp_path / "r")
        assert r.returncode == 2 and why in r.stderr, (name, r.stderr)


# ---- CPU: the shared wire-format module on its own -----------------------------

@pytest.fixture(scope="module")
def wire(tmp_path_factory):
    """tests/wire_format_check.cpp compiled against cli/wire_format.hpp."""
    exe = tmp_path_factory.mktemp("wire") / "wire_format_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                    f"-I{ROOT / 'reformulation_b200' / 'cli'}", str(HERE / "wire_format_check.cpp"),
                    "-o", str(exe)], check=True)
    return exe


def wire_json(exe, *args):
    r = run(exe, *args)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def test_wire_reads_what_numpy_writes(wire, tmp_path):
    q = qubo_sparse_bernoulli(4, 30, 0.2)
    write_praq(q, tmp_path / "q.bin")
    got = wire_json(wire, "qubo", tmp_path / "q.bin")
    assert got["ok"] and (got["n"], got["m"]) == (q.n, q.edges)
    assert np.array_equal(got["diag"], q.diag) and np.array_equal(got["vals"], q.vals)
    assert np.array_equal(got["rows"], q.rows) and np.array_equal(got["cols"], q.cols)
    j = jrp_demand(3, 3, 5)
    write_pria(j, tmp_path / "j.bin")
    got = wire_json(wire, "jrp", tmp_path / "j.bin")
    assert got["ok"] and (got["n"], got["t"], got["k0"]) == (3, 5, j.joint_order_cost)
    assert np.array_equal(got["k"], j.order_costs)
    assert np.array_equal(np.reshape(got["h"], (3, 5, 5)), j.holding_costs)
    edgeless = QuboInstance("e", "e", 3, np.array([1.0, -2.0, 0.5]), np.zeros(0, np.int64),
                            np.zeros(0, np.int64), np.zeros(0))
    write_praq(edgeless, tmp_path / "e.bin")
    got = wire_json(wire, "qubo", tmp_path / "e.bin")
    assert got["ok"] and got["m"] == 0 and got["rows"] == []


def test_wire_rejects_bad_files(wire, tmp_path):
    assert "cannot open" in wire_json(wire, "qubo", tmp_path / "missing")["error"]
    (tmp_path / "empty").write_bytes(b"")
    assert wire_json(wire, "jrp", tmp_path / "empty")["error"] == "file ends early"
    (tmp_path / "swap").write_bytes(struct.pack("<qqq", PRIA_MAGIC, 1, 1) + b"\0" * 24)
    assert "wrong magic" in wire_json(wire, "qubo", tmp_path / "swap")["error"]
    # a header claiming an overflowing payload is refused before any allocation
    (tmp_path / "over").write_bytes(struct.pack("<qqq", PRAQ_MAGIC, 1 << 62, 1 << 62))
    assert "size mismatch" in wire_json(wire, "qubo", tmp_path / "over")["error"]
    (tmp_path / "jover").write_bytes(struct.pack("<qqq", PRIA_MAGIC, 1 << 40, 1 << 40))
    assert "size mismatch" in wire_json(wire, "jrp", tmp_path / "jover")["error"]


def test_wire_record_layout_and_atomic_commit(wire, tmp_path):
    out = tmp_path / "r.bin"
    assert wire_json(wire, "record", out, "3", "17", "1", "--", "-2.5", "4.25", "--",
                     "0", "0.5", "1")["ok"]
    iters, status, lower, upper, x = read_praq(out)
    assert (iters, status, lower, upper) == (17, 1, -2.5, 4.25) and list(x) == [0, 0.5, 1]
    assert sorted(p.name for p in tmp_path.iterdir()) == ["r.bin"]       # no .partial left
    res = wire_json(wire, "record", tmp_path / "no" / "such" / "dir" / "r.bin", "1")
    assert not res["ok"] and "cannot create" in res["error"]


@pytest.mark.parametrize("argv,want", [
    (["a", "b"], dict(tolerance=None, max_iter=None, flags=[])),
    (["a", "b", "1e-6"], dict(tolerance=1e-6, max_iter=None, flags=[])),
    (["a", "b", "1e-6", "-1", "f32", "solution"], dict(tolerance=1e-6, max_iter=-1, flags=["f32", "solution"])),
    (["a", "b", "vanilla", "verbose"], dict(tolerance=None, max_iter=None, flags=["vanilla", "verbose"])),
    (["a", "b", "1e-4", "f32"], dict(tolerance=1e-4, max_iter=None, flags=["f32"])),
])
def test_wire_argument_parsing(wire, argv, want):
    got = wire_json(wire, "args", *argv)
    assert got["ok"] and {k: got[k] for k in want} == want


@pytest.mark.parametrize("argv,why", [
    (["a"], "missing"), (["a", "b", "0"], "positive"), (["a", "b", "-1e-4"], "positive"),
    (["a", "b", "nan"], "unexpected"), (["a", "b", "1e-4", "12x"], "unexpected"),
    (["a", "b", "1e-4", "5", "6"], "unexpected"), (["a", "b", "f64"], "unexpected"),
])
def test_wire_argument_errors(wire, argv, why):
    got = wire_json(wire, "args", *argv)
    assert not got["ok"] and why in got["error"]


def test_fixtures_written_by_the_reference_decode(wire):
    """The committed files of tests/golden/wire/ (written by the reference's own
    harness, tests/golden/make_wire_fixtures.py) decode to the instances they
    were made from."""
    q = qubo_sparse_bernoulli(0, 200, 0.05)
    got = wire_json(wire, "qubo", GOLDEN / "qubo_n200.bin")
    assert got["ok"] and np.array_equal(got["vals"], q.vals) and np.array_equal(got["rows"], q.rows)
    j = jrp_demand(7, 6, 20)
    got = wire_json(wire, "jrp", GOLDEN / "jrp_6x20.bin")
    assert got["ok"] and np.array_equal(np.reshape(got["h"], (6, 20, 20)), j.holding_costs)


# ---- CPU: the reference's own harness code against this library's files -------

REFERENCE = Path("/root/reference")
needs_reference = pytest.mark.skipif(not (REFERENCE / "qubo" / "harness").exists(),
                                     reason="the reference tree is not present on this machine")


def in_reference(project, code, **env_vars):
    """Run `code` with the reference project's `harness` package importable (a
    child process: both projects name their package `harness`); its stdout is
    one JSON line."""
    env = dict(os.environ, PYTHONPATH=f"{REFERENCE / project}{os.pathsep}{ROOT}", **env_vars)
    r = subprocess.run([sys.executable, "-c", textwrap.dedent(code)], capture_output=True,
                       text=True, timeout=300, cwd=str(ROOT), env=env)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


@needs_reference
def test_reference_harness_and_wire_module_agree(wire, tmp_path):
    """qubo/harness/backends/praq_cuda.py and jrp/harness/backends/pria_cuda.py
    write instances that the wire module reads back exactly, and read the
    records it writes."""
    got = in_reference("qubo", f"""
        import json
        from pathlib import Path
        from reformulation_b200.instances import qubo_uniform_edges
        from harness.backends.praq_cuda import write_instance
        write_instance(qubo_uniform_edges(5, 50, 120), Path({str(tmp_path / "q.bin")!r}))
        print(json.dumps(dict(ok=True)))""")
    assert got["ok"]
    q = wire_json(wire, "qubo", tmp_path / "q.bin")
    from reformulation_b200.instances import qubo_uniform_edges
    ref = qubo_uniform_edges(5, 50, 120)
    assert np.array_equal(q["vals"], ref.vals) and np.array_equal(q["cols"], ref.cols)
    wire_json(wire, "record", tmp_path / "r.bin", "4", "33", "0", "--", "-1.5", "2", "--",
              "0", "1", "0.5", "1")
    back = in_reference("qubo", f"""
        import json
        from pathlib import Path
        from harness.backends.praq_cuda import read_result
        it, st, lo, up, x = read_result(Path({str(tmp_path / "r.bin")!r}))
        print(json.dumps(dict(it=it, st=st, lo=lo, up=up, x=list(map(float, x)))))""")
    assert back == dict(it=33, st=0, lo=-1.5, up=2.0, x=[0.0, 1.0, 0.5, 1.0])
    in_reference("jrp", f"""
        import json
        from pathlib import Path
        from reformulation_b200.instances import jrp_demand
        from harness.backends.pria_cuda import write_instance
        write_instance(jrp_demand(9, 4, 7), Path({str(tmp_path / "j.bin")!r}))
        print(json.dumps(dict(ok=True)))""")
    j = wire_json(wire, "jrp", tmp_path / "j.bin")
    ref = jrp_demand(9, 4, 7)
    assert np.array_equal(np.reshape(j["h"], (4, 7, 7)), ref.holding_costs) and j["k0"] == ref.joint_order_cost
    wire_json(wire, "record", tmp_path / "s.bin", "4", "7", "96", "1", "--", "10.5", "11", "0.02")
    back = in_reference("jrp", f"""
        import json
        from pathlib import Path
        from harness.backends.pria_cuda import read_result
        print(json.dumps(read_result(Path({str(tmp_path / "s.bin")!r}))))""")
    assert back == [96, 1, 10.5, 11.0, 0.02]


@needs_reference
def test_reference_ctypes_libraries_bind_this_library(native):
    """The reference's in-process wrappers (qubo/harness/praq_cuda_library.py:
    90-139, jrp/harness/pria_cuda_library.py:82-132) load libreform_b200.so
    and read the same defaults and check intervals through their own struct
    definitions (host-only calls)."""
    from reformulation_b200 import build, praq, pria
    lib = str(build.LIB)
    got = in_reference("qubo", f"""
        import json
        from harness.praq_cuda_library import Library
        L = Library({lib!r})
        p = L.parameters(op_steps=0)
        print(json.dumps(dict(d=L.parameters().as_dict(),
                              iv=[L.check_interval(n, p) for n in (1000, 50000, 400000, 2000000)])))""")
    ours = praq.Library()
    mine = ours.parameters()
    assert got["d"] == {k: getattr(mine, k) for k, _ in mine._fields_}
    q0 = ours.parameters(op_steps=0)
    assert got["iv"] == [ours.check_interval(n, q0) for n in (1000, 50000, 400000, 2000000)]
    got = in_reference("jrp", f"""
        import json
        from harness.pria_cuda_library import Library
        p = Library({lib!r}).parameters(1e-5, 700)
        print(json.dumps({{k: getattr(p, k) for k, _ in p._fields_}}))""")
    mine = pria.Library().parameters(700, 1e-5)
    assert got == {k: getattr(mine, k) for k, _ in mine._fields_}


@needs_reference
def test_reference_backend_drives_the_cli(bins, tmp_path):
    """The reference's subprocess backend (qubo/harness/backends/praq_cuda.py:
    79-167), pointed at this CLI, runs it with its own arguments and reads its
    files.  With a device the solve is optimal; without one the CLI stops at
    device set-up (exit 3, no result file) and the backend reports an error
    with the CLI's reason."""
    import torch
    got = in_reference("qubo", f"""
        import json, math
        import harness.backends.praq_cuda as backend
        from harness.config import Tolerances
        from pathlib import Path
        from reformulation_b200.instances import qubo_sparse_bernoulli
        backend.praq_cuda_bin = lambda: Path({str(bins[0])!r})
        r = backend.solve(qubo_sparse_bernoulli(0, 200, 0.05), tolerances=Tolerances(optimality=1e-6),
                          time_limit=120.0)
        print(json.dumps(dict(status=r.status, note=r.note, objective=r.objective,
                              iterations=r.iterations, solve=r.solve_seconds)))""",
                       PRAQ_RESULTS_DIR=str(tmp_path))
    if torch.cuda.is_available():
        assert got["status"] == "optimal" and got["iterations"] > 0 and got["solve"] >= 0
    else:
        assert got["status"] == "error" and "no usable CUDA device" in got["note"]


# ---- GPU: results equal the C ABI's ---------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("f32", [False, True])
def test_praq_cli_equals_library(bins, tmp_path, f32):
    from reformulation_b200 import praq
    q = qubo_sparse_bernoulli(0, 200, 0.05)
    write_praq(q, tmp_path / "q.bin")
    tol = 1e-4 if f32 else 1e-6      # FP32 iterates level off near a 1e-6 gap
    args = [bins[0], tmp_path / "q.bin", tmp_path / "r.bin", str(tol), "0"] + (["f32"] if f32 else [])
    r = run(*args)
    assert r.returncode == 0, r.stderr
    iters, status, lower, upper, x = read_praq(tmp_path / "r.bin")
    lib = praq.Library()
    s = lib.solve(q, lib.parameters(tolerance=tol, use_float32=int(f32)))
    assert (iters, status, lower, upper) == (s.iterations, s.status, s.lower, s.upper)
    assert np.array_equal(x, s.x)
    k = keys(r.stdout)
    assert k["status"] == "converged" and int(k["iterations"]) == iters
    assert k["precision"] == ("float32" if f32 else "float64")
    assert float(k["solve_seconds"]) >= 0 and float(k["setup_seconds"]) >= 0


@pytest.mark.gpu
def test_praq_cli_iteration_limit(bins, tmp_path):
    q = qubo_sparse_bernoulli(3, 300, 0.05)
    write_praq(q, tmp_path / "q.bin")
    r = run(bins[0], tmp_path / "q.bin", tmp_path / "r.bin", "1e-12", "32")
    assert r.returncode == 1
    iters, status, lower, upper, _ = read_praq(tmp_path / "r.bin")
    assert status == 1 and iters == 32 and lower <= upper


@pytest.mark.gpu
@pytest.mark.parametrize("f32", [False, True])
def test_pria_cli_equals_library(bins, tmp_path, f32):
    from reformulation_b200 import pria
    j = jrp_demand(7, 6, 20)
    write_pria(j, tmp_path / "j.bin")
    tol = 1e-4 if f32 else 1e-6
    args = [bins[1], tmp_path / "j.bin", tmp_path / "r.bin", str(tol), "-1", "solution"] + (["f32"] if f32 else [])
    r = run(*args)
    assert r.returncode == 0, r.stderr
    out = read_pria(tmp_path / "r.bin", solution=True)
    # the CLI runs the device-resident API with FP64 input in both precisions
    with pria.DeviceSolver(j, pria.Library().parameters(-1, tol), "mixed" if f32 else "fp64") as dev:
        assert dev.run() == 0
        s = dev.result(want_solution=True)
    assert out["iterations"] == s.iterations and out["status"] == 0
    assert out["upper"] == s.primal_objective and out["lower"] == s.dual_objective
    assert np.array_equal(out["x"], s.x) and np.array_equal(out["z"], s.z)
    k = keys(r.stdout)
    assert (int(k["items"]), int(k["periods"])) == (6, 20) and k["status"] == "converged"
    assert k["precision"] == ("float32" if f32 else "float64") and k["method"] == "halpern"
    # without the flag only the 56-byte header is written
    r = run(bins[1], tmp_path / "j.bin", tmp_path / "r2.bin", str(tol), "-1", *(["f32"] if f32 else []))
    assert r.returncode == 0
    assert read_pria(tmp_path / "r2.bin")["iterations"] == out["iterations"]


@pytest.mark.gpu
def test_pria_cli_vanilla_and_verbose(bins, tmp_path):
    from reformulation_b200 import pria
    j = jrp_demand(8, 5, 14)
    write_pria(j, tmp_path / "j.bin")
    r = run(bins[1], tmp_path / "j.bin", tmp_path / "r.bin", "1e-12", "64", "vanilla", "verbose")
    assert r.returncode == 1, r.stderr          # the cap, not the gap, ended it
    out = read_pria(tmp_path / "r.bin")
    lib = pria.Library()
    s = lib.solve(j, lib.parameters(64, 1e-12, use_halpern=0))
    assert out["iterations"] == s.iterations == 64 and out["status"] == 1
    assert out["upper"] == s.primal_objective and out["lower"] == s.dual_objective
    assert "vanilla" in r.stderr                # per-check progress lines


@pytest.mark.gpu
def test_clis_on_files_written_by_the_reference_harness(bins, tmp_path):
    """The committed instance files written by the reference's own harness
    backends (tests/golden/make_wire_fixtures.py): each CLI solves them with
    the arguments the backends pass (<instance> <result> <tol>) and its result
    equals the library's solve of the same instance."""
    from reformulation_b200 import praq, pria
    r = run(bins[0], GOLDEN / "qubo_n200.bin", tmp_path / "q.out", "1e-6")
    assert r.returncode == 0, r.stderr
    iters, status, lower, upper, x = read_praq(tmp_path / "q.out")
    lib = praq.Library()
    s = lib.solve(qubo_sparse_bernoulli(0, 200, 0.05), lib.parameters(tolerance=1e-6))
    assert (iters, status, lower, upper) == (s.iterations, 0, s.lower, s.upper)
    assert np.array_equal(x, s.x)
    r = run(bins[1], GOLDEN / "jrp_6x20.bin", tmp_path / "j.out", "1e-6")
    assert r.returncode == 0, r.stderr
    out = read_pria(tmp_path / "j.out")
    with pria.DeviceSolver(jrp_demand(7, 6, 20), pria.Library().parameters(-1, 1e-6)) as dev:
        assert dev.run() == 0
        js = dev.result()
    assert (out["iterations"], out["status"]) == (js.iterations, 0)
    assert (out["lower"], out["upper"]) == (js.dual_objective, js.primal_objective)
    assert {"setup_seconds", "solve_seconds"} <= set(keys(r.stdout))
