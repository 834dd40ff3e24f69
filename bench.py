#!/usr/bin/env python
"""bench.py -- solves/s of the restarted Halpern PDHG hot path on B200.

Headline workload (one "step" = one full solve from the cold start):
    PRAQ, the QUBO roof-dual LP of a graph with n = 100,000 nodes and
    m = 1,000,000 distinct uniform pairs (seed 1), integer weights in
    [-100, 100], solved to 1e-4 relative gap (= relative KKT: both iterates
    are feasible by construction), FP32 iterates with FP64 reductions /
    restart logic / bounds ("mixed").  The plain FP64 kernel on the same
    instance is timed beside it.

The same JSON line carries one sub-object per other workload, each with its
own value, plain-FP64 comparator, roofline of its dominant kernel and CPU
baseline (at N = 1 only; rank 0):
    praq_n200      n = 200 QUBO (pairs kept with probability 0.05, seed 0):
                   latency p50/p99, device-resident and through praq_solve
    praq_n2e6      n = 2,000,000, m = 20,000,000 QUBO (seed 1), the largest
                   rung of the reference's own QUBO ladder: the HBM-bound size
    pria           JRP LP, N = 100 items, T = 500 periods (seed 2)
    batch          256 QUBO + 128 JRP of log-uniform sizes (seed 3) in one
                   batched engine, autotuned, per size class against plain FP64
    serving        Poisson arrivals, 70 % QUBO / 30 % JRP (seed 4), a short
                   sweep; `--workload serving` runs the long one

Timing: W untimed warm-up solves, then exactly K timed solves, each between a
CUDA event pair on the solver's stream (torch's current stream, passed down the
C ABI), with L2 flushed (a 256 MB write) before every solve and outside the
event pair; barrier + synchronize on both sides; max over ranks.  `value` is
whole-job solves/s.  `e2e` is the same metric through the reference-facing C
call praq_solve with host buffers (host->device upload of the instance and
device->host copy of the result inside the timed region).

Multi-GPU: instances are independent, so N GPUs run N replicas (weak scaling,
no collective on the data path); torch.distributed/NCCL only carries the
barrier and the max-over-ranks reduction of the timings.  `--gpus N` without
torchrun starts the N ranks itself.

--impl reference: the reference's CPU implementation of this path is its JAX
specification, which cannot run here (no jax); the arm times the CPU
restatement of it (oracle/praq_oracle.c, all host threads) on the same
workload, rank 0 only.

--profile-case {praq,pria}: one capped solve of a chosen size and nothing else
(the command the ncu summaries under profiles/ were taken with).
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "solves/sec and p50/p99 latency at 1e-4 rel KKT vs plain FP64 PDHG, 1 B200"
UNIT = "solves/s"
TOL = 1e-4
N_NODES, N_EDGES, SEED = 100_000, 1_000_000, 1
WORKLOAD = ("PRAQ QUBO roof-dual LP, n=100000 nodes, m=1000000 uniform distinct pairs "
            "(seed 1), weights U{-100..100}, solve to 1e-4 relative gap")
L2_NOTE = "flushed before every solve (256 MB write, outside the timed events)"


def peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def praq_bytes(n: int, m: int, real: int, index: int = 4) -> dict:
    """Per-launch algorithmic bytes of the two PRAQ step kernels.  The
    per-iteration total is n (6R + I) + m (11R + 4I): the node kernel reads x
    (predicted), x0, diag, deg and the CSR pointer and writes x, r
    (n (6R + I)) and reads the CSR index and one gathered dual per half-edge
    (m (2I + 2R)); the edge kernel reads both ends, the weight, the predicted
    dual pair, the anchor pair and r at both ends and writes the dual pair
    (m (2I + 9R))."""
    node = n * (6 * real + index) + m * (2 * index + 2 * real)
    edge = m * (2 * index + 9 * real)
    return {"node": node, "edge": edge, "node_check": node, "edge_check": edge,
            "iteration": node + edge}


def pria_bytes(nd: int, real: int) -> dict:
    """Per-launch algorithmic bytes of the PRIA half-steps (15 ND R per
    iteration): x reads x, x0, h, y, z and writes x, r (7 ND R); the y/z step
    reads y, y0, z, z0 and r twice and writes y, z (8 ND R)."""
    return {"x": 7 * nd * real, "yz": 8 * nd * real, "x_check": 7 * nd * real,
            "yz_check": 8 * nd * real, "iteration": 15 * nd * real}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 50 ms into a file."""

    FIELDS = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self, bus_id: str | None):
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            if bus_id and bus_id.lower() not in parts[0].lower() and parts[0].lower() not in bus_id.lower():
                continue
            try:
                rows.append(dict(sm=float(parts[1]), max=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], pcap=parts[8]))
            except ValueError:
                continue
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [r for r in rows if r["power"] > 200.0] or rows
        reasons = set()
        for r in loaded:
            if r["hw"] == "Active":
                reasons.add("hw_slowdown")
            if r["hwt"] == "Active":
                reasons.add("hw_thermal_slowdown")
            if r["swt"] == "Active":
                reasons.add("sw_thermal_slowdown")
            if r["pcap"] == "Active":
                reasons.add("sw_power_cap")
        return {"sm_mhz": statistics.median(r["sm"] for r in loaded),
                "sm_max_mhz": max(r["max"] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows), "samples_under_load": len(loaded)}


def read_traffic(profile: str, kind: str):
    """DRAM bytes per launch of `kind` from a committed ncu summary, if any
    (lines `traffic_bytes_per_launch <kind> <bytes>`)."""
    path = ROOT / "profiles" / profile
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kind:
            return float(parts[2])
    return None


def roofline(kind_label: str, alg_bytes: float, per_launch_ms: float, profile: str | None = None,
             kind: str | None = None, bound: str = "hbm") -> dict:
    peak, peak_kind = peaks()
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    return {"bound": bound, "kernel": kind_label, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "frac_of_8tbs": achieved / 8000.0,
            "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_us": per_launch_ms * 1e3,
            "traffic": read_traffic(profile, kind) if profile and kind else None}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0))


def cpu_leg(inst, threads: int, budget_s: float = 20.0, max_solves: int = 20, tol: float = TOL):
    """The oracle (CPU restatement of the reference's JAX solver), FP64, full
    solves to `tol` until `budget_s` of CPU time or `max_solves`."""
    import oracle
    p = oracle.praq_params(tolerance=tol)
    times, iters = [], []
    t_begin = time.perf_counter()
    while len(times) < max_solves and (time.perf_counter() - t_begin) < budget_s:
        t0 = time.perf_counter()
        r = oracle.praq_solve(inst, p, threads=threads)
        times.append(time.perf_counter() - t0)
        iters.append(r["iterations"])
    return times, iters


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    from reformulation_b200.instances import qubo_uniform_edges
    inst = qubo_uniform_edges(SEED, N_NODES, N_EDGES)
    threads = cpu_threads()
    # warm-up: page in the oracle and the instance
    cpu_leg(inst, threads, budget_s=0.0, max_solves=max(1, min(args.warmup, 1)))
    times, iters = cpu_leg(inst, threads, budget_s=1e9, max_solves=args.steps)
    total = sum(times)
    value = len(times) / total
    sample = (f"{len(times)} full solves of the workload to 1e-4 (FP64, {iters[0]} iterations), "
              f"CPU restatement oracle/praq_oracle.c with {threads} OpenMP threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64 (CPU)", "l2": "n/a (CPU)"},
        "p50_ms": 1e3 * float(np.percentile(times, 50)), "p99_ms": 1e3 * float(np.percentile(times, 99)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference's CPU implementation of this path is its JAX solver "
                 "(qubo/praq-jax), which cannot run without jax; this arm times the CPU "
                 "restatement of it"),
    }
    print(json.dumps(line), flush=True)
    return 0


class Timer:
    """CUDA-event timing of solves on one stream, L2 flushed before each."""

    def __init__(self, torch, stream, flush):
        self.torch, self.stream, self.flush = torch, stream, flush

    def solves(self, run, steps: int) -> list[float]:
        torch = self.torch
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for k in range(steps):
            self.flush.zero_()
            starts[k].record(self.stream)
            run()
            ends[k].record(self.stream)
        torch.cuda.synchronize()
        return [s.elapsed_time(e) for s, e in zip(starts, ends)]


def pct(values, q):
    return float(np.percentile(values, q)) if len(values) else math.nan


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


# ---- sub-objects (N = 1, rank 0) ----------------------------------------------

def sub_praq_n200(timer, steps, skip_cpu):
    """Config 1: the n = 200 QUBO, latency-bound.  Device-resident solves
    (event-timed) and solves through praq_solve with host buffers (wall
    clock), FP64 (the configuration's precision) and mixed."""
    from reformulation_b200 import praq
    from reformulation_b200.instances import qubo_sparse_bernoulli
    inst = qubo_sparse_bernoulli(0, 200, 0.05)
    lib = praq.Library()
    out = {"workload": "PRAQ n=200, pairs kept with probability 0.05 (seed 0), to 1e-4", "unit": UNIT}
    stream = timer.stream.cuda_stream
    for prec, f32 in (("fp64", 0), ("mixed", 1)):
        p = lib.parameters(tolerance=TOL, use_float32=f32)
        with praq.DeviceSolver(inst, p, stream=stream) as dev:
            # the per-kernel graph first, for comparison; then the automatic
            # choice (the persistent kernel at this size)
            dev.set_megakernel(0)
            for _ in range(5):
                dev.run()
            gms = timer.solves(dev.run, steps)
            graph = {"p50_ms": pct(gms, 50), "p99_ms": pct(gms, 99), "launches_per_solve": dev.launches()}
            persistent = dev.set_megakernel(-1)
            for _ in range(5):
                dev.run()
            ms = timer.solves(dev.run, steps)
            launches = dev.launches()
            res = dev.result(want_x=False)
            _, prof = dev.run_profiled()
        e2e = []
        for _ in range(steps):
            t0 = time.perf_counter()
            s = lib.solve(inst, p)
            e2e.append(time.perf_counter() - t0)
        assert s.status == 0
        alg = praq_bytes(inst.n, inst.edges, 8 if prec == "fp64" else 4)["iteration"]
        out[prec] = {"solves_per_s": 1e3 * len(ms) / sum(ms), "p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99),
                     "persistent_kernel": persistent, "launches_per_solve": launches, "graph": graph,
                     "e2e_solves_per_s": len(e2e) / sum(e2e), "e2e_p50_ms": 1e3 * pct(e2e, 50),
                     "e2e_p99_ms": 1e3 * pct(e2e, 99), "iterations": res.iterations,
                     "upper": res.upper, "relative_gap": res.gap,
                     "kernel_ms": {k: v[0] for k, v in prof.items() if v[1]}}
        out[prec]["achieved_gbs_whole_solve"] = alg * res.iterations / (pct(ms, 50) / 1e3) / 1e9
    out["value"] = out["mixed"]["solves_per_s"]
    out["plain_fp64"] = {"value": out["fp64"]["solves_per_s"], "p50_ms": out["fp64"]["p50_ms"],
                         "p99_ms": out["fp64"]["p99_ms"]}
    out["roofline"] = {"bound": "latency", "note": "30 KB of iterates: one CTA's dependency latency "
                       "bound (the persistent kernel is a grid of one CTA here), not HBM; "
                       "achieved_gbs_whole_solve gives bytes per second of a solve",
                       "achieved": out["mixed"]["achieved_gbs_whole_solve"], "peak": peaks()[0],
                       "unit": "GB/s", "frac": out["mixed"]["achieved_gbs_whole_solve"] / peaks()[0]}
    if not skip_cpu:
        times, iters = cpu_leg(inst, 1, budget_s=2.0, max_solves=200)
        out["cpu_baseline"] = {"value": len(times) / sum(times), "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"{len(times)} FP64 solves to 1e-4 ({iters[0]} iterations) by "
                                         "the CPU restatement oracle/praq_oracle.c, 1 thread",
                               "p50_ms": 1e3 * pct(times, 50)}
        import oracle
        ref = oracle.praq_solve(inst, oracle.praq_params(tolerance=TOL))
        out["objective_check"] = {
            "oracle_fp64_upper": ref["upper"], "oracle_iterations": ref["iterations"],
            "fp64_rel_err": rel(out["fp64"]["upper"], ref["upper"]),
            "mixed_rel_err": rel(out["mixed"]["upper"], ref["upper"]),
            "maxflow_roof_dual": oracle.roof_dual_maxflow(inst)}
    return out


def sub_praq_n2e6(timer, steps, skip_cpu):
    """The reference's top QUBO rung: n = 2,000,000, m = 20,000,000 (uniform
    pairs, seed 1), to 1e-4; the working set (1.3 GB in FP32) is far above L2,
    so this is the HBM-bound size."""
    from reformulation_b200 import praq
    from reformulation_b200.instances import qubo_uniform_edges
    n, m = 2_000_000, 20_000_000
    inst = qubo_uniform_edges(1, n, m)
    lib = praq.Library()
    out = {"workload": "PRAQ n=2000000, m=20000000 uniform distinct pairs (seed 1), to 1e-4",
           "unit": UNIT, "l2": L2_NOTE}
    stream = timer.stream.cuda_stream
    for prec, f32 in (("mixed", 1), ("fp64", 0)):
        p = lib.parameters(tolerance=TOL, use_float32=f32)
        with praq.DeviceSolver(inst, p, stream=stream) as dev:
            for _ in range(3):
                dev.run()
            ms = timer.solves(dev.run, steps)
            res = dev.result(want_x=False)
            _, prof = dev.run_profiled()
        kinds = {k: v for k, v in prof.items() if v[1]}
        dom = max(kinds, key=lambda k: kinds[k][0])
        real = 4 if f32 else 8
        out[prec] = {"solves_per_s": 1e3 * len(ms) / sum(ms), "ms_per_solve": sum(ms) / len(ms),
                     "p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99), "iterations": res.iterations,
                     "upper": res.upper, "lower": res.lower, "relative_gap": res.gap,
                     "kernels_ms_per_launch": {k: v[0] / v[1] for k, v in kinds.items()},
                     "kernels_share": {k: v[0] / sum(x[0] for x in kinds.values()) for k, v in kinds.items()},
                     "roofline": roofline(f"praq {dom} kernel ({'fp32' if f32 else 'fp64'})",
                                          praq_bytes(n, m, real)[dom], kinds[dom][0] / kinds[dom][1],
                                          "praq_edge_node_n2M_m20M.txt" if f32 else None, dom)}
    out["value"] = out["mixed"]["solves_per_s"]
    out["plain_fp64"] = {"value": out["fp64"]["solves_per_s"], "p50_ms": out["fp64"]["p50_ms"]}
    out["roofline"] = out["mixed"]["roofline"]
    out["mixed_vs_fp64_upper_rel"] = rel(out["mixed"]["upper"], out["fp64"]["upper"])
    if not skip_cpu:
        threads = cpu_threads()
        times, iters = cpu_leg(inst, threads, budget_s=1.0, max_solves=1)
        out["cpu_baseline"] = {"value": len(times) / sum(times), "unit": UNIT, "cores": threads,
                               "kind": "port",
                               "sample": f"one FP64 solve to 1e-4 ({iters[0]} iterations) by the CPU "
                                         f"restatement oracle/praq_oracle.c, {threads} OpenMP threads"}
        out["objective_check"] = {"oracle_fp64_iterations": iters[0]}
    return out


def sub_pria(timer, steps, skip_cpu):
    """Config 3: one JRP LP, N = 100 items, T = 500 periods (seed 2), to 1e-4,
    mixed beside plain FP64; one step = one solve from the cold start on the
    resident instance."""
    from reformulation_b200 import pria
    from reformulation_b200.instances import jrp_demand
    items, periods = 100, 500
    inst = jrp_demand(2, items, periods)
    nd = items * periods * (periods + 1) // 2
    lib = pria.Library()
    out = {"workload": "PRIA JRP LP N=100 T=500 (seed 2), demand-driven H, to 1e-4", "unit": UNIT,
           "l2": L2_NOTE}
    stream = timer.stream.cuda_stream
    for prec in ("mixed", "fp64"):
        with pria.DeviceSolver(inst, lib.parameters(1_000_000, TOL), prec, stream=stream) as dev:
            for _ in range(2):
                dev.run()
            ms = timer.solves(dev.run, steps)
            r = dev.result()
            _, prof = dev.run_profiled()
        kinds = {k: v for k, v in prof.items() if v[1]}
        dom = max(("x", "yz"), key=lambda k: kinds[k][0])
        real = 4 if prec == "mixed" else 8
        per = {k: v[0] / v[1] for k, v in kinds.items()}
        alg = pria_bytes(nd, real)
        out[prec] = {"solves_per_s": 1e3 * len(ms) / sum(ms), "ms_per_solve": sum(ms) / len(ms),
                     "p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99), "iterations": r.iterations,
                     "relative_gap": r.relative_gap, "upper": r.primal_objective,
                     "lower": r.dual_objective, "kernels_ms_per_launch": per,
                     "kernels_share": {k: v[0] / sum(x[0] for x in kinds.values()) for k, v in kinds.items()},
                     "x_kernel_gbs": alg["x"] / (per["x"] / 1e3) / 1e9,
                     "yz_kernel_gbs": alg["yz"] / (per["yz"] / 1e3) / 1e9,
                     "roofline": roofline(f"pria {dom} half-step ({'fp32' if real == 4 else 'fp64'})",
                                          alg[dom], per[dom], "pria_x_y_z_N100_T500.txt" if real == 4 else None,
                                          dom)}
    # end to end through pria_solve_f32: the instance held as float32 host
    # arrays (K, H), as that entry point takes it, and the three solution
    # arrays (N x T x T each) out, set-up and tear-down included; one untimed
    # solve first
    params = lib.parameters(1_000_000, TOL)
    inst32 = dataclasses.replace(inst, order_costs=inst.order_costs.astype(np.float32),
                                 holding_costs=inst.holding_costs.astype(np.float32))
    e2e = []
    for k in range(4):
        t0 = time.perf_counter()
        s = lib.solve(inst32, params, "f32", want_solution=True)
        if k:
            e2e.append(time.perf_counter() - t0)
        assert s.status == 0
    out["e2e"] = {"value": len(e2e) / sum(e2e), "unit": UNIT, "p50_ms": 1e3 * pct(e2e, 50),
                  "h2d_bytes_per_step": 4 * (inst.order_costs.size + inst.holding_costs.size),
                  "d2h_bytes_per_step": 3 * 4 * items * periods * periods,
                  "form": "pria_solve_f32 on float32 host arrays, with the solution arrays"}
    out["value"] = out["mixed"]["solves_per_s"]
    out["plain_fp64"] = {"value": out["fp64"]["solves_per_s"], "p50_ms": out["fp64"]["p50_ms"]}
    out["roofline"] = out["mixed"]["roofline"]
    out["mixed_vs_fp64"] = out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
    out["mixed_vs_fp64_upper_rel"] = rel(out["mixed"]["upper"], out["fp64"]["upper"])
    if not skip_cpu:
        import oracle
        threads = cpu_threads()
        block = 16
        t0 = time.perf_counter()
        oracle.pria_solve(inst, oracle.pria_params(max_iter=block, tolerance=TOL), threads=threads)
        t_block = time.perf_counter() - t0
        iters = out["fp64"]["iterations"]
        est = t_block / block * iters
        out["cpu_baseline"] = {"value": 1.0 / est, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"{block} iterations (one check block, set-up included) of the "
                                         f"FP64 CPU restatement oracle/pria_oracle.c, {threads} OpenMP "
                                         f"threads, {t_block:.2f} s, scaled to the {iters} iterations of "
                                         "a full solve"}
    return out


def sub_pria_small(timer, steps, skip_cpu):
    """Small JRPs, latency-bound: N=10, T=25 and N=30, T=75 (seeds 5, 6), to
    1e-4.  Device-resident solves from the cold start with the solver's
    automatic choice beside the per-kernel graph and the persistent kernel
    (one cooperative launch per check block) forced on, mixed and FP64;
    solves through pria_solve with host buffers; the CPU restatement on one
    thread."""
    from reformulation_b200 import pria
    from reformulation_b200.instances import jrp_demand
    lib = pria.Library()
    stream = timer.stream.cuda_stream
    out = {"workload": "PRIA JRP LP N=10 T=25 (seed 5) and N=30 T=75 (seed 6), demand-driven H, to 1e-4",
           "unit": UNIT}
    for n, t, seed in ((10, 25, 5), (30, 75, 6)):
        inst = jrp_demand(seed, n, t)
        p = lib.parameters(1_000_000, TOL)
        rec = {"entries": inst.entries}
        for prec in ("mixed", "fp64"):
            for mode, name in ((-1, "auto"), (0, "graph"), (1, "persistent")):
                with pria.DeviceSolver(inst, p, prec, stream=stream) as dev:
                    active = dev.set_megakernel(mode)
                    for _ in range(3):
                        dev.run()
                    ms = timer.solves(dev.run, steps)
                    r = dev.result()
                    launches = dev.launches()
                rec[f"{prec}_{name}"] = {
                    "persistent_kernel": active, "solves_per_s": 1e3 * len(ms) / sum(ms),
                    "p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99), "iterations": r.iterations,
                    "upper": r.primal_objective, "relative_gap": r.relative_gap,
                    "launches_per_solve": launches}
        e2e = []
        for _ in range(steps):
            t0 = time.perf_counter()
            s = lib.solve(inst, p, precision="mixed")
            e2e.append(time.perf_counter() - t0)
            assert s.status == 0
        rec["mixed_e2e"] = {"solves_per_s": len(e2e) / sum(e2e), "p50_ms": 1e3 * pct(e2e, 50),
                            "p99_ms": 1e3 * pct(e2e, 99)}
        rec["graph_over_persistent_p50"] = {
            prec: rec[f"{prec}_graph"]["p50_ms"] / rec[f"{prec}_persistent"]["p50_ms"] for prec in ("mixed", "fp64")}
        rec["mixed_vs_fp64_upper_rel"] = rel(rec["mixed_auto"]["upper"], rec["fp64_auto"]["upper"])
        if not skip_cpu:
            import oracle
            tt = []
            while sum(tt) < 2.0 and len(tt) < 50:
                t0 = time.perf_counter()
                ref = oracle.pria_solve(inst, oracle.pria_params(tolerance=TOL), threads=1)
                tt.append(time.perf_counter() - t0)
            rec["cpu_baseline"] = {"value": len(tt) / sum(tt), "unit": UNIT, "cores": 1, "kind": "port",
                                   "sample": f"{len(tt)} FP64 solves to 1e-4 ({ref['iterations']} iterations) "
                                             "by the CPU restatement oracle/pria_oracle.c, 1 thread",
                                   "p50_ms": 1e3 * pct(tt, 50)}
            rec["objective_check"] = {"oracle_fp64_upper": ref["upper"],
                                      "fp64_rel_err": rel(rec["fp64_auto"]["upper"], ref["upper"]),
                                      "mixed_rel_err": rel(rec["mixed_auto"]["upper"], ref["upper"])}
        out[f"n{n}_t{t}"] = rec
    big = out["n30_t75"]
    out["value"] = big["mixed_auto"]["solves_per_s"]
    out["plain_fp64"] = {"value": big["fp64_auto"]["solves_per_s"], "p50_ms": big["fp64_auto"]["p50_ms"]}
    if "cpu_baseline" in big:
        out["cpu_baseline"] = big["cpu_baseline"]
    out["roofline"] = {"bound": "latency", "note": "under 2 MB of iterates, L2-resident: launch, barrier and "
                       "dependency latency bound, not HBM"}
    return out


def _size_class(kind: str, inst) -> str:
    if kind == "qubo":
        n = inst.n
        return "qubo n<2k" if n < 2000 else ("qubo 2k<=n<10k" if n < 10_000 else "qubo n>=10k")
    nd = inst.entries
    return "jrp ND<1M" if nd < 1_000_000 else ("jrp 1M<=ND<10M" if nd < 10_000_000 else "jrp ND>=10M")


def sub_batch(timer, steps, warmup, skip_cpu, qubos=256, jrps=128, autotune=True, fp64_stride=1,
              rep=None):
    """Config 4: 256 QUBO + 128 JRP of log-uniform sizes (seed 3) in one
    batched engine (FP32 iterates, FP64 reductions; a QUBO that stalls in FP32
    continues in FP64), to 1e-4; one step = a cold restart and a full solve of
    every instance, resident on the device.  The comparator is the plain FP64
    single-instance solver on every instance in turn (device-resident, one
    warm run then a timed run).  Per size class: the class alone in a batch
    against the same FP64 solves.

    With `rep` spanning N > 1 ranks the instances are routed over the GPUs
    (replicas.route on replicas.work_estimate); each rank runs its share in
    its own engine, the step time is the slowest rank's, and `value` is all
    instances over it (strong scaling: the batch is fixed); the comparator,
    the class breakdown and the CPU sample are N = 1 measurements and are left
    out."""
    from reformulation_b200 import praq, pria
    from reformulation_b200.batch import EscalatingBatch
    from reformulation_b200.instances import batch_mix
    torch = timer.torch
    stream = timer.stream
    t_gen = time.perf_counter()
    qs, js = batch_mix(3, qubos, jrps)
    t_gen = time.perf_counter() - t_gen
    ql, jl = praq.Library(), pria.Library()
    qp = ql.parameters(tolerance=TOL, max_iter=1_000_000, use_float32=1)
    jp = jl.parameters(1_000_000, TOL)
    items = [("qubo", q) for q in qs] + [("jrp", j) for j in js]
    world = rep.world if rep is not None else 1
    n_all = len(items)
    if world > 1:
        from reformulation_b200.replicas import route, work_estimate
        mine = route([work_estimate(x) for _, x in items], world)[rep.rank]
        items = [items[k] for k in mine]

    def engine(subset):
        b = EscalatingBatch(stream=stream.cuda_stream)
        ids = [b.add_qubo(x, qp) if k == "qubo" else b.add_jrp_demand(x, jp) for k, x in subset]
        b.start()
        return b, ids

    def timed(b, nsteps):
        ms = []
        for _ in range(nsteps):
            b.restart()
            timer.flush.zero_()
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            b.run()
            e.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(e))
        return ms

    t_lay = time.perf_counter()
    b, ids = engine(items)
    t_lay = time.perf_counter() - t_lay
    shapes = b.b32.autotune() if autotune else None
    for _ in range(warmup):
        b.restart()
        b.run()
    launches0 = b.launches()
    if world > 1:
        rep.barrier()
    ms = timed(b, steps)
    launches = b.launches() - launches0
    if world > 1:
        rep.barrier()
        step_max = rep.max(sum(ms) / len(ms))
        b.close()
        return {"workload": f"batch {len(qs)} QUBO + {len(js)} JRP (seed 3), to 1e-4, routed over "
                            f"{world} GPUs", "value": 1e3 * n_all / step_max, "unit": UNIT,
                "scaling": "strong", "n_gpus": world, "ms_per_step": step_max, "steps": steps,
                "instances": n_all, "instances_this_rank": len(items), "shapes": shapes,
                "gpu_launches_this_rank": int(launches)}
    its, gaps, alg, uppers = [], [], 0.0, []
    for (kind, x), i in zip(items, ids):
        done, it, lo, up = b.status(i)
        its.append(it)
        uppers.append(up)
        gaps.append((up - lo) / (1 + abs(up) + abs(lo)))
        alg += it * (praq_bytes(x.n, x.edges, 4)["iteration"] if kind == "qubo"
                     else pria_bytes(x.entries, 4)["iteration"])
    escalated = len(b.escalated)
    dev_bytes = b.device_bytes()
    b.close()
    total = len(items)
    step_ms = sum(ms) / len(ms)
    value = 1e3 * total / step_ms

    # plain FP64, one instance at a time
    # (and the same single-instance solver with FP32 iterates, to split the
    # batch's gain into precision and batching)
    fp64_ms, fp64_upper, mixed_ms, mixed_capped = {}, {}, {}, []
    for k, (kind, x) in enumerate(items):
        if k % fp64_stride:
            continue
        dense = x if kind == "qubo" else x.build()
        for prec in ("fp64", "mixed"):
            # (FP32 iterates alone level off near a 1e-3 gap on a few hard QUBOs,
            # which the batch moves to FP64; alone they stop at 20,000 iterations)
            if kind == "qubo":
                dev = praq.DeviceSolver(dense, ql.parameters(tolerance=TOL,
                                                             max_iter=1_000_000 if prec == "fp64" else 20_000,
                                                             use_float32=int(prec == "mixed")),
                                        stream=stream.cuda_stream)
            else:
                dev = pria.DeviceSolver(dense, jl.parameters(1_000_000, TOL), prec,
                                        stream=stream.cuda_stream)
            dev.run()
            t_ms = timer.solves(dev.run, 1)[0]
            if prec == "fp64":
                fp64_ms[k] = t_ms
                r64 = dev.result()
                fp64_upper[k] = r64.upper if kind == "qubo" else r64.primal_objective
            else:
                mixed_ms[k] = t_ms
                r32 = dev.result()
                g32 = r32.gap if kind == "qubo" else r32.relative_gap
                if not g32 <= TOL:
                    mixed_capped.append(k)
            dev.close()
    fp64_value = 1e3 * len(fp64_ms) / sum(fp64_ms.values())
    diffs = [rel(uppers[k], fp64_upper[k]) for k in fp64_upper]

    # per size class: the class alone in a batch, against its FP64 solves
    classes = {}
    for k, (kind, x) in enumerate(items):
        classes.setdefault(_size_class(kind, x), []).append(k)
    per_class = {}
    for name, ks in sorted(classes.items()):
        cb, cids = engine([items[k] for k in ks])
        if shapes:
            cb.b32.set_shapes(shapes["grid_multiplier"])
        cb.run()
        cms = timed(cb, 1)[0]
        calg = sum(cb.status(i)[1] * (praq_bytes(items[k][1].n, items[k][1].edges, 4)["iteration"]
                                      if items[k][0] == "qubo" else pria_bytes(items[k][1].entries, 4)["iteration"])
                   for k, i in zip(ks, cids))
        cb.close()
        f64 = [fp64_ms[k] for k in ks if k in fp64_ms]
        f32 = [mixed_ms[k] for k in ks if k in mixed_ms and k not in mixed_capped]
        per_class[name] = {"instances": len(ks), "batched_ms": cms, "batched_solves_per_s": 1e3 * len(ks) / cms,
                           "plain_fp64_ms": sum(f64), "plain_fp64_solves_per_s": 1e3 * len(f64) / sum(f64),
                           "single_mixed_ms": sum(f32),
                           "batched_vs_plain_fp64": (1e3 * len(ks) / cms) / (1e3 * len(f64) / sum(f64)),
                           "achieved_gbs": calg / (cms / 1e3) / 1e9}
    peak = peaks()
    out = {"workload": f"batch {len(qs)} QUBO + {len(js)} JRP (seed 3), to 1e-4", "value": value,
           "unit": UNIT, "steps": steps, "warmup": warmup, "ms_per_step": step_ms,
           "dtype": "f32 iterates, f64 reductions", "l2": L2_NOTE, "instances": total,
           "max_gap": max(gaps), "iterations_p50": pct(its, 50), "iterations_max": int(max(its)),
           "device_bytes": dev_bytes, "shapes": shapes, "escalated_to_fp64": escalated,
           "gpu_launches": int(launches),
           "plain_fp64": {"value": fp64_value, "unit": UNIT, "sample": len(fp64_ms),
                          "ms_total": sum(fp64_ms.values()),
                          "note": "every instance solved alone by the FP64 single-instance solver, "
                                  "device-resident, event-timed"},
           "batched_vs_plain_fp64": value / fp64_value,
           "single_mixed": {"value": 1e3 * len(mixed_ms) / sum(mixed_ms.values()), "unit": UNIT,
                            "not_converged": len(mixed_capped),
                            "value_converged_only": 1e3 * (len(mixed_ms) - len(mixed_capped)) / max(
                                1e-9, sum(v for k, v in mixed_ms.items() if k not in mixed_capped)),
                            "note": "every instance solved alone with FP32 iterates and no escalation "
                                    "(device-resident); QUBOs that level off stop at 20,000 iterations"},
           "objective_vs_plain_fp64": {
               "max_rel": max(diffs), "median_rel": pct(diffs, 50),
               "above_1e-6": int(sum(d > 1e-6 for d in diffs)), "instances": len(diffs),
               "note": "each instance's batched FP32-iterate objective (upper bound) against the "
                       "plain FP64 single-instance solve, both to a 1e-4 gap"},
           "per_class": per_class,
           "roofline": {"bound": "hbm", "kernel": "all batched kernels over a whole step",
                        "achieved": alg / (step_ms / 1e3) / 1e9, "peak": peak[0], "unit": "GB/s",
                        "frac": alg / (step_ms / 1e3) / 1e9 / peak[0], "peak_kind": peak[1],
                        "algorithmic_bytes_per_step": alg, "traffic": None,
                        "note": "sum over instances of iterations x per-iteration algorithmic bytes "
                                "(FP32 sizes), over the step time"},
           "generate_s": t_gen, "layout_s": t_lay}
    if not skip_cpu:
        import oracle
        threads = cpu_threads()
        sample, t_cpu, budget = [], 0.0, 15.0
        for k in range(0, total, 16):
            kind, x = items[k]
            if kind == "jrp" and x.entries > 2_000_000:
                continue
            t0 = time.perf_counter()
            if kind == "qubo":
                oracle.praq_solve(x, oracle.praq_params(tolerance=TOL), threads=threads)
            else:
                oracle.pria_solve(x.build(), oracle.pria_params(tolerance=TOL), threads=threads)
            t_cpu += time.perf_counter() - t0
            sample.append(k)
            if t_cpu > budget:
                break
        gpu_same = sum(fp64_ms[k] for k in sample if k in fp64_ms) / 1e3
        out["cpu_baseline"] = {"value": len(sample) / t_cpu, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"every 16th instance of the batch (JRPs above 2M entries "
                                         f"left out), {len(sample)} FP64 solves to 1e-4 by the CPU "
                                         f"restatements oracle/praq_oracle.c and oracle/pria_oracle.c, "
                                         f"{threads} OpenMP threads",
                               "same_sample_plain_fp64_gpu_solves_per_s": len(sample) / gpu_same if gpu_same else None}
    return out


def sub_serving(rates, seconds, warm_s, pool_qubo=28, pool_jrp=12, tol=TOL, admit_every=None):
    """Config 5: Poisson arrivals (seed 4) at each rate for `seconds` after a
    `warm_s` warm-up stream, 70 % QUBO / 30 % JRP, instances drawn from a pool
    of the batch workload's size distributions; device-memory admission budget
    150 GB.  Latency = arrival to result on the host.  The plain-FP64
    comparator is simulated: the same arrival stream served FIFO by one
    plain FP64 solver, from each pool instance's measured end-to-end time."""
    from reformulation_b200 import serving
    from reformulation_b200.instances import _jrp_log_uniform, _qubo_log_uniform
    rng = np.random.default_rng(4)
    pool_q = [_qubo_log_uniform(rng, k, 4) for k in range(pool_qubo)]
    pool_j = [_jrp_log_uniform(rng, k, 4) for k in range(pool_jrp)]
    svc = serving.service_times_fp64(pool_q + pool_j, tol)
    svc_q, svc_j = svc[:len(pool_q)], svc[len(pool_q):]

    def stream_of(rate, horizon, seed):
        arr = np.random.default_rng(seed)
        reqs, service, t, k = [], [], 0.0, 0
        while True:
            t += float(arr.exponential(1.0 / rate))
            if t > horizon:
                break
            if arr.random() < 0.7:
                idx = int(arr.integers(len(pool_q)))
                reqs.append(serving.Request(k, t, pool_q[idx]))
                service.append(svc_q[idx])
            else:
                idx = int(arr.integers(len(pool_j)))
                reqs.append(serving.Request(k, t, pool_j[idx]))
                service.append(svc_j[idx])
            k += 1
        return reqs, service

    rows = []
    for rate in rates:
        server = serving.Server(budget_bytes=150e9, tolerance=tol,
                                **({"admit_every": admit_every} if admit_every else {}))
        if warm_s > 0:
            warm, _ = stream_of(rate, warm_s, 40)
            server.serve(warm)
            server.done.clear()
        reqs, service = stream_of(rate, seconds, 4)
        done = server.serve(reqs)
        wall = max(c.finished for c in done) if done else math.nan
        lat = [c.latency for c in done]
        seq = serving.sequential_fifo([r.arrival for r in reqs], service)
        free = 0.0
        for a, s in sorted(zip([r.arrival for r in reqs], service)):
            free = max(a, free) + s
        rows.append({"rate": rate, "requests": len(reqs), "completed": len(done),
                     "solves_per_s": len(done) / wall,
                     **{f"{q}_ms": 1e3 * v for q, v in serving.percentiles(lat).items()},
                     "max_gap": max(c.gap for c in done), "hbm_high_water_gb": server.high_water / 1e9,
                     "plain_fp64_fifo_simulated": {
                         "solves_per_s": len(reqs) / free,
                         **{f"{q}_ms": 1e3 * v for q, v in serving.percentiles(seq).items()}}})
        server.close()
    return {"workload": "serving: Poisson arrivals, 70% QUBO / 30% JRP (seed 4)", "unit": UNIT,
            "seconds_per_rate": seconds, "warmup_seconds": warm_s,
            "pool": {"qubo": len(pool_q), "jrp": len(pool_j)}, "rates": rows,
            "value": max(r["solves_per_s"] for r in rows),
            "plain_fp64": {"value": max(r["plain_fp64_fifo_simulated"]["solves_per_s"] for r in rows),
                           "note": "simulated FIFO from measured per-instance end-to-end FP64 times"}}


# ---- the default line ----------------------------------------------------------

def run_ours(args):
    import torch

    from reformulation_b200 import build as native_build
    from reformulation_b200 import praq
    from reformulation_b200.instances import qubo_uniform_edges
    from reformulation_b200.replicas import Replicas

    world, rank, local = dist_setup()
    if world > 1 and world != args.gpus:
        raise SystemExit(f"WORLD_SIZE={world} but --gpus {args.gpus}")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    rep = Replicas("nccl", device=device)
    native_build.build()
    stream = torch.cuda.current_stream(device)
    barrier, max_over_ranks = rep.barrier, rep.max

    inst = qubo_uniform_edges(SEED, N_NODES, N_EDGES)
    lib = praq.Library()
    p_mixed = lib.parameters(tolerance=TOL, use_float32=1, max_iter=1_000_000)
    p_fp64 = lib.parameters(tolerance=TOL, use_float32=0, max_iter=1_000_000)
    mixed = praq.DeviceSolver(inst, p_mixed, stream=stream.cuda_stream)
    fp64 = praq.DeviceSolver(inst, p_fp64, stream=stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    timer = Timer(torch, stream, flush)

    for _ in range(args.warmup):
        mixed.run()
        fp64.run()
    torch.cuda.synchronize()

    sampler = ClockSampler()
    if rank == 0:
        sampler.start()
    barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    statuses, launches = [], []

    def one():
        statuses.append(mixed.run())
        launches.append(mixed.launches())    # kernel launches of that run (graph nodes counted)

    ms = timer.solves(one, args.steps)
    torch.cuda.synchronize()
    barrier()
    wall = time.perf_counter() - wall0
    if rank == 0:
        sampler.stop()
    res = mixed.result()
    total_ms = max_over_ranks(sum(ms))
    value = world * args.steps / (total_ms / 1e3)

    # the plain FP64 kernel on the same instance, same protocol
    barrier()
    ms64 = timer.solves(fp64.run, args.steps)
    barrier()
    res64 = fp64.result()
    total64 = max_over_ranks(sum(ms64))
    value64 = world * args.steps / (total64 / 1e3)

    # live per-kernel timing (event pair around every launch of one solve)
    _, prof = mixed.run_profiled()
    kinds = {k: v for k, v in prof.items() if v[1] > 0}
    dominant = max(kinds, key=lambda k: kinds[k][0])
    alg = praq_bytes(N_NODES, N_EDGES, 4)
    _, prof64 = fp64.run_profiled()
    alg64 = praq_bytes(N_NODES, N_EDGES, 8)
    k64 = max((k for k, v in prof64.items() if v[1]), key=lambda k: prof64[k][0])

    # e2e through the reference-facing C call, host buffers; the same W
    # untimed warm-up calls first (the first one-shot solves of a process pay
    # for the memory pool's growth and the like)
    for _ in range(args.warmup):
        assert lib.solve(inst, p_mixed).status == 0
    barrier()
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        s = lib.solve(inst, p_mixed)
        e2e_times.append(time.perf_counter() - t0)
        assert s.status == 0
    barrier()
    e2e_total = max_over_ranks(sum(e2e_times))
    e2e_value = world * args.steps / e2e_total
    n, m = N_NODES, N_EDGES
    # praq_solve uploads diag (f64) and rows, cols (int64) and vals (f64) as
    # given; it reads back the primal (FP32 iterates) and one control block
    # per check
    h2d = 8 * n + 24 * m
    blocks = res.iterations // 16 + 2
    d2h = n * 4 + 96 * (blocks + 2)

    line = None
    if rank == 0:
        props = torch.cuda.get_device_properties(device)
        bus = None
        if all(hasattr(props, a) for a in ("pci_domain_id", "pci_bus_id", "pci_device_id")):
            bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}"
        clocks = sampler.summary(bus)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 iterates, f64 reductions", "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "mixed (fp32 iterates / fp64 reductions)",
                       "parallelism": f"replicas x{world}", "l2": L2_NOTE},
            "p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99),
            "iterations": res.iterations, "relative_gap": res.gap, "lower": res.lower,
            "upper": res.upper, "statuses_ok": all(s == 0 for s in statuses),
            "plain_fp64": {"value": value64, "unit": UNIT, "ms_per_step": total64 / args.steps,
                           "p50_ms": pct(ms64, 50), "p99_ms": pct(ms64, 99),
                           "iterations": res64.iterations, "relative_gap": res64.gap,
                           "upper": res64.upper,
                           "kernels_ms_per_launch": {k: v[0] / v[1] for k, v in prof64.items() if v[1]},
                           "dominant_kernel": k64,
                           "dominant_kernel_gbs": alg64[k64] / (prof64[k64][0] / prof64[k64][1] / 1e3) / 1e9},
            "mixed_vs_fp64": value / value64,
            "roofline": roofline(f"praq {dominant} kernel (fp32)", alg.get(dominant),
                                 kinds[dominant][0] / kinds[dominant][1], "praq_kernels_n100k_m1M.txt",
                                 dominant),
            "kernels_ms_per_launch": {k: v[0] / v[1] for k, v in kinds.items()},
            "kernels_share": {k: v[0] / sum(x[0] for x in kinds.values()) for k, v in kinds.items()},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "p50_ms": 1e3 * pct(e2e_times, 50),
                    "p99_ms": 1e3 * pct(e2e_times, 99), "max_ms": 1e3 * max(e2e_times)},
            "gpu_launches": int(sum(launches)),
            "clocks": clocks,
            "wall_s_timed_region": wall,
        }

    if rank == 0 and not args.skip_cpu:
        import oracle
        flow = oracle.roof_dual_maxflow(inst)
        line["objective_check"] = {
            "maxflow_roof_dual": flow,
            "mixed_upper_rel_err": rel(res.upper, flow),
            "fp64_upper_rel_err": rel(res64.upper, flow),
            "mixed_vs_fp64_upper_rel": rel(res.upper, res64.upper),
            "brackets_contain_optimum": bool(res.lower <= flow + 1e-9 * abs(flow) <= res.upper + 2e-9 * abs(flow)
                                             and res64.lower <= flow + 1e-9 * abs(flow) <= res64.upper + 2e-9 * abs(flow))}

    # CPU baseline and the reference's own praq-cuda, rank 0 at N=1 only
    if rank == 0 and world == 1 and not args.skip_cpu:
        threads = cpu_threads()
        times, iters = cpu_leg(inst, threads, budget_s=20.0, max_solves=10)
        line["cpu_baseline"] = {
            "value": len(times) / sum(times), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"{len(times)} full FP64 solves of the workload to 1e-4 ({iters[0]} "
                       f"iterations each) by the CPU restatement oracle/praq_oracle.c, "
                       f"{threads} OpenMP threads")}
        import oracle
        ref = oracle.praq_solve(inst, oracle.praq_params(tolerance=TOL), threads=threads)
        line["objective_check"]["oracle_fp64"] = {
            "iterations": ref["iterations"], "upper": ref["upper"], "lower": ref["lower"],
            "gpu_fp64_upper_rel": rel(res64.upper, ref["upper"]),
            "gpu_fp64_lower_rel": rel(res64.lower, ref["lower"]),
            "gpu_mixed_upper_rel": rel(res.upper, ref["upper"])}
        try:
            rp = oracle.RefPraq()
            ref_rows = {}
            for prec in (0, 1):
                rp.solve(inst, tolerance=TOL, use_float32=prec)
                tt = []
                for _ in range(3):
                    t0 = time.perf_counter()
                    rr = rp.solve(inst, tolerance=TOL, use_float32=prec)
                    tt.append(time.perf_counter() - t0)
                ref_rows["f32" if prec else "f64"] = {
                    "solves_per_s_e2e": 3 / sum(tt), "iterations": rr["iterations"],
                    "upper": rr["upper"]}
            line["reference_praq_cuda_same_gpu"] = ref_rows
        except Exception as exc:  # the reference build is optional context
            line["reference_praq_cuda_same_gpu"] = {"unavailable": str(exc)[:120]}
    mixed.close()
    fp64.close()

    # the other workloads, one GPU
    if rank == 0 and world == 1 and not args.headline_only:
        sub_steps = max(3, min(args.steps, 10))
        for key, fn in (("praq_n200", lambda: sub_praq_n200(timer, 50, args.skip_cpu)),
                        ("praq_n2e6", lambda: sub_praq_n2e6(timer, sub_steps, args.skip_cpu)),
                        ("pria", lambda: sub_pria(timer, sub_steps, args.skip_cpu)),
                        ("pria_small", lambda: sub_pria_small(timer, 30, args.skip_cpu)),
                        ("batch", lambda: sub_batch(timer, 3, 2, args.skip_cpu)),
                        ("serving", lambda: sub_serving([50, 100], 8.0, 2.0))):
            t0 = time.perf_counter()
            try:
                line[key] = fn()
            except Exception as exc:   # one workload's failure must not hide the others'
                line[key] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
            line[key]["bench_wall_s"] = time.perf_counter() - t0

    if rank == 0:
        print(json.dumps(line), flush=True)
    rep.close()
    return 0


# ---- the single-workload modes -------------------------------------------------

def _single(args, key, fn):
    """One workload alone.  Under torchrun only `batch` uses every rank (its
    instances routed over the GPUs); the others run on rank 0."""
    import torch
    from reformulation_b200 import build as native_build
    from reformulation_b200.replicas import Replicas
    world, rank, local = dist_setup()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    rep = Replicas("nccl", device=device)
    native_build.build()
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    out = None
    if key == "batch" or rank == 0:
        out = fn(Timer(torch, stream, flush), rep)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "n_gpus": world, "data": "synthetic", key: out}), flush=True)
    rep.close()
    return 0


def run_profile_case(args):
    """One capped solve of a chosen size, for ncu (see profiles/)."""
    from reformulation_b200 import build as native_build
    native_build.build()
    if args.profile_case == "praq":
        from reformulation_b200 import praq
        from reformulation_b200.instances import qubo_uniform_edges
        inst = qubo_uniform_edges(args.seed, args.n, args.m)
        lib = praq.Library()
        p = lib.parameters(tolerance=args.tol, max_iter=args.max_iter,
                           use_float32=int(args.precision == "mixed"))
        with praq.DeviceSolver(inst, p) as dev:
            t0 = time.perf_counter()
            st = dev.run()
            dt = time.perf_counter() - t0
            r = dev.result(want_x=False)
        print(f"praq n={args.n} m={args.m} status={st} iterations={r.iterations} "
              f"lower={r.lower:.10g} upper={r.upper:.10g} seconds={dt:.4f}")
        return 0 if st >= 0 else 1
    from reformulation_b200 import pria
    from reformulation_b200.instances import jrp_demand
    inst = jrp_demand(args.seed, args.items, args.periods)
    res = pria.solve_arrays(inst, tolerance=args.tol, max_iter=args.max_iter, precision=args.precision)
    print(f"pria N={args.items} T={args.periods} status={res['status']} iterations={res['iterations']} "
          f"lower={res['lower']:.10g} upper={res['upper']:.10g}")
    return 0 if res["status"] in (0, -1) else 1


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_ranks(argv: list[str], gpus: int) -> int:
    """`--gpus N` without torchrun: start the N ranks here (one per GPU) and
    return the launcher's status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(Path(__file__).resolve()), *argv]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU baseline legs")
    ap.add_argument("--headline-only", action="store_true", help="omit the sub-objects")
    ap.add_argument("--workload", choices=("default", "praq_n200", "praq_n2e6", "pria", "pria_small", "batch",
                                           "serving"),
                    default="default", help="one workload alone (longer settings than the default line)")
    ap.add_argument("--qubos", type=int, default=256)
    ap.add_argument("--jrps", type=int, default=128)
    ap.add_argument("--fp64-stride", type=int, default=1)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--rates", type=float, nargs="+", default=[50, 100, 200, 500, 1000, 2000])
    ap.add_argument("--seconds", type=float, default=60.0)
    ap.add_argument("--warm-seconds", type=float, default=5.0)
    ap.add_argument("--admit-every", type=int, default=None,
                    help="serving: blocks between admissions while requests run")
    ap.add_argument("--profile-case", choices=("praq", "pria"))
    ap.add_argument("--n", type=int, default=100_000)
    ap.add_argument("--m", type=int, default=1_000_000)
    ap.add_argument("--items", type=int, default=100)
    ap.add_argument("--periods", type=int, default=500)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--max-iter", type=int, default=64)
    ap.add_argument("--tol", type=float, default=TOL)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="mixed")
    args = ap.parse_args()
    if args.profile_case:
        return run_profile_case(args)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(sys.argv[1:], args.gpus)
    if args.impl == "reference":
        args.warmup = max(args.warmup, 3)
        return run_reference(args)
    if args.workload == "praq_n200":
        return _single(args, "praq_n200", lambda t, rep: sub_praq_n200(t, args.steps, args.skip_cpu))
    if args.workload == "praq_n2e6":
        return _single(args, "praq_n2e6", lambda t, rep: sub_praq_n2e6(t, args.steps, args.skip_cpu))
    if args.workload == "pria":
        return _single(args, "pria", lambda t, rep: sub_pria(t, args.steps, args.skip_cpu))
    if args.workload == "pria_small":
        return _single(args, "pria_small", lambda t, rep: sub_pria_small(t, args.steps, args.skip_cpu))
    if args.workload == "batch":
        return _single(args, "batch", lambda t, rep: sub_batch(t, args.steps, max(args.warmup, 1),
                                                               args.skip_cpu, args.qubos, args.jrps,
                                                               not args.no_autotune, args.fp64_stride, rep))
    if args.workload == "serving":
        return _single(args, "serving", lambda t, rep: sub_serving(args.rates, args.seconds,
                                                                   args.warm_seconds,
                                                                   admit_every=args.admit_every))
    args.warmup = max(args.warmup, 3)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
