"""The file CLIs praq_solve_file / pria_solve_file, which the reference's
harness backends drive as subprocesses (qubo/harness/backends/praq_cuda.py:27-86,
jrp/harness/backends/pria_cuda.py).  The instance/result wire formats, the
flags and the exit codes are the contract of qubo/praq-cuda/tools/
praq_solve_file.cu:7-31 and jrp/pria-cuda/tools/pria_solve_file.cu:7-45.

CPU tests: every exit-2 path (usage, unreadable or malformed input), which is
reached before any CUDA call.  GPU tests: a solve through the CLI equals the
same solve through the C ABI bit for bit (bounds, iterations, x), the stdout
"key: value" lines the harness parses, the solution flag and the f32 flag.
"""

import struct
import subprocess

import numpy as np
import pytest

from reformulation_b200.instances import jrp_demand, qubo_sparse_bernoulli

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
    assert run(pria).returncode == 2
    assert run(praq, tmp_path / "missing", tmp_path / "r").returncode == 2
    assert run(pria, tmp_path / "missing", tmp_path / "r").returncode == 2
    inst = tmp_path / "i"
    inst.write_bytes(b"")
    assert run(pria, inst, tmp_path / "r", "1e-4", "-1", "bogus").returncode == 2


def test_malformed_files_are_rejected(bins, tmp_path):
    praq, pria = bins
    q = qubo_sparse_bernoulli(0, 20, 0.3)
    good = tmp_path / "q.bin"
    write_praq(q, good)
    raw = good.read_bytes()
    for name, data in (("magic", struct.pack("<q", 7) + raw[8:]), ("short", raw[:-8]),
                       ("negative", raw[:8] + struct.pack("<q", -1) + raw[16:])):
        f = tmp_path / name
        f.write_bytes(data)
        r = run(praq, f, tmp_path / "r")
        assert r.returncode == 2 and "not a PRAQ instance" in r.stderr
        assert not (tmp_path / "r").exists()
    j = jrp_demand(1, 2, 4)
    pj = tmp_path / "j.bin"
    write_pria(j, pj)
    raw = pj.read_bytes()
    for name, data in (("jmagic", struct.pack("<q", PRAQ_MAGIC) + raw[8:]), ("jshort", raw[:-8]),
                       ("jzero", raw[:8] + struct.pack("<q", 0) + raw[16:])):
        f = tmp_path / name
        f.write_bytes(data)
        r = run(pria, f, tmp_path / "r")
        assert r.returncode == 2 and "not a PRIA instance" in r.stderr


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
    lib = pria.Library()
    s = lib.solve(j, lib.parameters(-1, tol), precision="mixed" if f32 else "fp64", want_solution=True)
    assert out["iterations"] == s.iterations and out["status"] == 0
    assert out["upper"] == s.primal_objective and out["lower"] == s.dual_objective
    assert np.array_equal(out["x"], s.x.astype(np.float64))
    assert np.array_equal(out["z"], s.z.astype(np.float64))
    k = keys(r.stdout)
    assert (int(k["items"]), int(k["periods"])) == (6, 20) and k["status"] == "converged"
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
