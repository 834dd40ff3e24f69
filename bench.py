#!/usr/bin/env python
"""bench.py -- solves/s of the restarted Halpern PDHG hot path on B200.

Workload (one "step" = one full solve from the cold start):
    PRAQ, the QUBO roof-dual LP of a graph with n = 100,000 nodes and
    m = 1,000,000 distinct uniform pairs (seed 1), integer weights in
    [-100, 100], solved to 1e-4 relative gap (= relative KKT: both iterates
    are feasible by construction), FP32 iterates with FP64 reductions /
    restart logic / bounds ("mixed").  The plain FP64 kernel on the same
    instance is timed beside it.

Timing: W untimed warm-up solves, then exactly K timed solves, each between a
CUDA event pair on the solver's stream (torch's current stream, passed down the
C ABI), with L2 flushed (a 256 MB write) before every solve and outside the
event pair; barrier + synchronize on both sides; max over ranks.  `value` is
whole-job solves/s.  `e2e` is the same metric through the reference-facing C
call praq_solve with host buffers (host layout build, host->device upload and
device->host result inside the timed region).

Multi-GPU: PRAQ instances are independent, so N GPUs run N replicas (weak
scaling, no collective on the data path); torch.distributed/NCCL only carries
the barrier and the max-over-ranks reduction of the timings.

--impl reference: the reference's CPU implementation of this path is its JAX
specification, which cannot run here (no jax); the arm times the CPU
restatement of it (oracle/praq_oracle.c, all host threads) on the same
workload, rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import math
import os
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


def peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(n: int, m: int, real: int, index: int = 4) -> dict:
    """Per-launch algorithmic bytes of the two step kernels.  The per-iteration
    total is the PRAQ figure n (6R + I) + m (11R + 4I): the node kernel reads
    x (predicted), x0, diag, deg and the CSR pointer and writes x, r
    (n (6R + I)) and reads the CSR index and one gathered dual per half-edge
    (m (2I + 2R)); the edge kernel reads both ends, the weight, the predicted
    dual pair, the anchor pair and r at both ends and writes the dual pair
    (m (2I + 9R))."""
    node = n * (6 * real + index) + m * (2 * index + 2 * real)
    edge = m * (2 * index + 9 * real)
    return {"node": node, "edge": edge, "node_check": node, "edge_check": edge,
            "iteration": node + edge}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 50 ms into a file."""

    FIELDS = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        self.t0 = self.t1 = None

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


def read_traffic(kind: str):
    """dram bytes per launch of `kind` from the committed ncu summary, if any."""
    path = ROOT / "profiles" / "praq_kernels_n100k_m1M.txt"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kind:
            return float(parts[2])
    return None


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0))


def cpu_leg(inst, threads: int, budget_s: float = 20.0, max_solves: int = 20):
    """The oracle (CPU restatement of the reference's JAX solver), FP64, full
    solves to 1e-4 until `budget_s` of CPU time or `max_solves`."""
    import oracle
    p = oracle.praq_params(tolerance=TOL)
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


def time_solves(dev, steps, flush, torch, stream):
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    launches = 0
    statuses = []
    for k in range(steps):
        flush.zero_()
        starts[k].record(stream)
        statuses.append(dev.run())
        ends[k].record(stream)
        launches += dev.launches()
    torch.cuda.synchronize()
    ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    return ms, launches, statuses


def run_ours(args):
    import torch

    from reformulation_b200 import build as native_build
    from reformulation_b200 import praq
    from reformulation_b200.instances import qubo_uniform_edges

    from reformulation_b200.replicas import Replicas

    world, rank, local = dist_setup()
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
    ms, launches, statuses = time_solves(mixed, args.steps, flush, torch, stream)
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
    ms64, _, st64 = time_solves(fp64, args.steps, flush, torch, stream)
    barrier()
    res64 = fp64.result()
    total64 = max_over_ranks(sum(ms64))
    value64 = world * args.steps / (total64 / 1e3)

    # live per-kernel timing (event pair around every launch of one solve)
    _, prof = mixed.run_profiled()
    kinds = {k: v for k, v in prof.items() if v[1] > 0}
    dominant = max(kinds, key=lambda k: kinds[k][0])
    per_launch_ms = kinds[dominant][0] / kinds[dominant][1]
    alg = algorithmic_bytes(N_NODES, N_EDGES, 4)
    hbm_peak, peak_kind = peaks()
    achieved = alg.get(dominant, 0) / (per_launch_ms / 1e3) / 1e9
    _, prof64 = fp64.run_profiled()
    alg64 = algorithmic_bytes(N_NODES, N_EDGES, 8)
    k64 = max((k for k, v in prof64.items() if v[1]), key=lambda k: prof64[k][0])

    # e2e through the reference-facing C call, host buffers
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
    h2d = 2 * (n + 1) * 4 + m * 4 + m * 8 + m * 4 + 3 * n * 4
    blocks = res.iterations // 16 + 2
    d2h = n * 4 + 96 * (blocks + 2)

    line = None
    if rank == 0:
        props = torch.cuda.get_device_properties(device)
        bus = None
        if all(hasattr(props, a) for a in ("pci_domain_id", "pci_bus_id", "pci_device_id")):
            bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}"
        clocks = sampler.summary(bus)
        lat = np.array(ms)
        lat64 = np.array(ms64)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 iterates, f64 reductions", "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "mixed (fp32 iterates / fp64 reductions)",
                       "parallelism": f"replicas x{world}",
                       "l2": "flushed before every solve (256 MB write, outside the timed events)"},
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "iterations": res.iterations, "relative_gap": res.gap, "lower": res.lower,
            "upper": res.upper, "statuses_ok": all(s == 0 for s in statuses),
            "plain_fp64": {"value": value64, "unit": UNIT, "ms_per_step": total64 / args.steps,
                           "p50_ms": float(np.percentile(lat64, 50)),
                           "p99_ms": float(np.percentile(lat64, 99)),
                           "iterations": res64.iterations, "relative_gap": res64.gap,
                           "upper": res64.upper,
                           "kernels_ms_per_launch": {k: v[0] / v[1] for k, v in prof64.items() if v[1]},
                           "dominant_kernel": k64,
                           "dominant_kernel_gbs": alg64[k64] / (prof64[k64][0] / prof64[k64][1] / 1e3) / 1e9},
            "mixed_vs_fp64": value / value64,
            "roofline": {"bound": "hbm", "kernel": f"praq {dominant} kernel (fp32)",
                         "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "peak_kind": peak_kind,
                         "frac_of_8tbs": achieved / 8000.0,
                         "algorithmic_bytes_per_launch": alg.get(dominant),
                         "avg_launch_us": per_launch_ms * 1e3,
                         "traffic": read_traffic(dominant)},
            "kernels_ms_per_launch": {k: v[0] / v[1] for k, v in kinds.items()},
            "kernels_share": {k: v[0] / sum(x[0] for x in kinds.values()) for k, v in kinds.items()},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "p50_ms": 1e3 * float(np.percentile(e2e_times, 50))},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "wall_s_timed_region": wall,
        }

    # the objective against the exact roof dual (max-flow) and the FP64 run
    if rank == 0 and not args.skip_cpu:
        import oracle
        flow = oracle.roof_dual_maxflow(inst)
        line["objective_check"] = {
            "maxflow_roof_dual": flow,
            "mixed_upper_rel_err": abs(res.upper - flow) / (1.0 + abs(flow)),
            "fp64_upper_rel_err": abs(res64.upper - flow) / (1.0 + abs(flow)),
            "mixed_vs_fp64_upper_rel": abs(res.upper - res64.upper) / (1.0 + abs(res64.upper)),
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
        try:
            import oracle
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

    if rank == 0:
        print(json.dumps(line), flush=True)
    mixed.close()
    fp64.close()
    rep.close()
    return 0


def _timed_events(torch, stream):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_pria(args):
    """Config 3: one JRP LP, N = 100 items, T = 500 periods (seed 2), to 1e-4,
    mixed precision beside plain FP64; one step = one solve from the cold
    start on the resident instance."""
    import torch

    from reformulation_b200 import pria
    from reformulation_b200.instances import jrp_demand

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    inst = jrp_demand(2, 100, 500)
    lib = pria.Library()
    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for prec in ("mixed", "fp64"):
        dev = pria.DeviceSolver(inst, lib.parameters(1_000_000, TOL), prec, stream=stream.cuda_stream)
        for _ in range(args.warmup):
            dev.run()
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            a, b = _timed_events(torch, stream)
            a.record(stream)
            dev.run()
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        r = dev.result()
        _, prof = dev.run_profiled()
        real = 4 if prec == "mixed" else 8
        nd = 100 * 500 * 501 // 2
        per = {k: v[0] / v[1] for k, v in prof.items() if v[1]}
        out[prec] = {"solves_per_s": 1e3 * len(ms) / sum(ms), "p50_ms": float(np.percentile(ms, 50)),
                     "p99_ms": float(np.percentile(ms, 99)), "iterations": r.iterations,
                     "relative_gap": r.relative_gap, "upper": r.primal_objective,
                     "kernels_ms_per_launch": per,
                     "x_kernel_gbs": 7 * nd * real / (per["x"] / 1e3) / 1e9,
                     "yz_kernel_gbs": 8 * nd * real / (per["yz"] / 1e3) / 1e9}
        dev.close()
    line = {"metric": METRIC, "workload": "PRIA JRP LP N=100 T=500 (seed 2), demand-driven H, to 1e-4",
            "value": out["mixed"]["solves_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "mixed": out["mixed"], "plain_fp64": out["fp64"],
            "mixed_vs_fp64": out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"],
            "mixed_objective_rel_err_vs_fp64": abs(out["mixed"]["upper"] - out["fp64"]["upper"])
                                               / (1.0 + abs(out["fp64"]["upper"])),
            "peak_hbm_gbs": peaks()[0], "data": "synthetic"}
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """Config 4: 256 QUBO + 128 JRP of log-uniform sizes (seed 3) in one
    engine, mixed precision, to 1e-4; one step = a cold restart and a full
    solve of all 384 instances, resident on the device.  The plain FP64
    single-instance kernel is timed on every instance (each solved alone,
    device-resident; `--fp64-stride` k > 1 takes every k-th one, a quicker but
    noisy estimate, since a few large JRPs carry most of the time)."""
    import torch

    from reformulation_b200 import praq, pria
    from reformulation_b200.batch import EscalatingBatch
    from reformulation_b200.instances import batch_mix

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    t_gen = time.perf_counter()
    qs, js = batch_mix(3, args.qubos, args.jrps)
    t_gen = time.perf_counter() - t_gen
    ql, jl = praq.Library(), pria.Library()
    qp = ql.parameters(tolerance=TOL, max_iter=1_000_000, use_float32=1)
    jp = jl.parameters(1_000_000, TOL)
    b = EscalatingBatch(stream=stream.cuda_stream)
    t_lay = time.perf_counter()
    ids = [b.add_qubo(q, qp) for q in qs] + [b.add_jrp_demand(j, jp) for j in js]
    b.start()
    t_lay = time.perf_counter() - t_lay
    shapes = b.b32.autotune() if args.autotune else None
    for _ in range(args.warmup):
        b.restart()
        b.run()
    ms = []
    launches0 = b.launches()
    for _ in range(args.steps):
        b.restart()
        a, e = _timed_events(torch, stream)
        a.record(stream)
        b.run()
        e.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(e))
    launches = b.launches() - launches0
    its = []
    gaps = []
    for i in ids:
        done, it, lo, up = b.status(i)
        its.append(it)
        gaps.append((up - lo) / (1 + abs(up) + abs(lo)))
    total = len(ids)
    value = 1e3 * total * len(ms) / sum(ms)
    # plain FP64 single-instance kernel on a sample
    sample = list(range(0, total, args.fp64_stride))
    fp64_ms = []
    for k in sample:
        if k < len(qs):
            dev = praq.DeviceSolver(qs[k], ql.parameters(tolerance=TOL, max_iter=1_000_000),
                                    stream=stream.cuda_stream)
        else:
            dev = pria.DeviceSolver(js[k - len(qs)].build(), jl.parameters(1_000_000, TOL), "fp64",
                                    stream=stream.cuda_stream)
        dev.run()
        a, e = _timed_events(torch, stream)
        a.record(stream)
        dev.run()
        e.record(stream)
        torch.cuda.synchronize()
        fp64_ms.append(a.elapsed_time(e))
        dev.close()
    fp64_value = 1e3 * len(fp64_ms) / sum(fp64_ms)
    line = {"metric": METRIC, "workload": f"batch {len(qs)} QUBO + {len(js)} JRP (seed 3), to 1e-4",
            "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sum(ms) / len(ms), "dtype": "f32 iterates, f64 reductions",
            "instances": total, "max_gap": max(gaps), "iterations_p50": float(np.percentile(its, 50)),
            "iterations_max": int(max(its)), "device_bytes": b.device_bytes(), "shapes": shapes,
            "escalated_to_fp64": len(b.escalated),
            "gpu_launches": int(launches),
            "plain_fp64_sequential": {"value": fp64_value, "unit": UNIT, "sample": len(sample),
                                      "sample_stride": args.fp64_stride},
            "batched_vs_plain_fp64": value / fp64_value,
            "generate_s": t_gen, "layout_s": t_lay, "data": "synthetic"}
    b.close()
    print(json.dumps(line), flush=True)
    return 0


def run_serving(args):
    """Config 5: Poisson arrivals (seed 4) at each rate of --rates for
    --seconds, 70 % QUBO / 30 % JRP, instances drawn from a pool of the
    config-4 size distributions; HBM admission budget 150 GB.  Latency =
    arrival to result on the host.  Comparator: the same arrival stream served
    FIFO by the plain FP64 single-instance solver (its measured end-to-end time
    per pool instance)."""
    import torch

    from reformulation_b200 import serving
    from reformulation_b200.instances import _jrp_log_uniform, _qubo_log_uniform

    torch.cuda.set_device(0)
    rng = np.random.default_rng(4)
    pool_q = [_qubo_log_uniform(rng, k, 4) for k in range(args.pool_qubo)]
    pool_j = [_jrp_log_uniform(rng, k, 4) for k in range(args.pool_jrp)]
    svc = serving.service_times_fp64(pool_q + pool_j, TOL)
    svc_q, svc_j = svc[:len(pool_q)], svc[len(pool_q):]
    rows = []
    for rate in args.rates:
        arr = np.random.default_rng(4)
        reqs, kinds, t = [], [], 0.0
        k = 0
        while True:
            t += float(arr.exponential(1.0 / rate))
            if t > args.seconds:
                break
            if arr.random() < 0.7:
                idx = int(arr.integers(len(pool_q)))
                reqs.append(serving.Request(k, t, pool_q[idx]))
                kinds.append(svc_q[idx])
            else:
                idx = int(arr.integers(len(pool_j)))
                reqs.append(serving.Request(k, t, pool_j[idx]))
                kinds.append(svc_j[idx])
            k += 1
        server = serving.Server(budget_bytes=150e9, tolerance=TOL)
        t0 = time.perf_counter()
        done = server.serve(reqs, t0=t0)
        wall = max(c.finished for c in done) if done else 0.0
        lat = [c.latency for c in done]
        seq = serving.sequential_fifo([r.arrival for r in reqs], kinds)
        seq_wall = max(r.arrival for r in reqs) + 0.0
        free = 0.0
        for a, s in sorted(zip([r.arrival for r in reqs], kinds)):
            free = max(a, free) + s
        rows.append({"rate": rate, "requests": len(reqs), "solves_per_s": len(done) / wall,
                     **{f"{q}_ms": 1e3 * v for q, v in serving.percentiles(lat).items()},
                     "max_gap": max(c.gap for c in done), "hbm_high_water_gb": server.high_water / 1e9,
                     "plain_fp64_fifo": {"solves_per_s": len(reqs) / free,
                                         **{f"{q}_ms": 1e3 * v for q, v in serving.percentiles(seq).items()}}})
        server.close()
        del seq_wall
    line = {"metric": METRIC, "workload": "serving: Poisson arrivals, 70% QUBO / 30% JRP (seed 4)",
            "unit": UNIT, "n_gpus": 1, "seconds_per_rate": args.seconds,
            "pool": {"qubo": len(pool_q), "jrp": len(pool_j)}, "rates": rows, "data": "synthetic"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU baseline leg")
    ap.add_argument("--workload", choices=("praq", "pria", "batch", "serving"), default="praq",
                    help="praq (the default line); pria, batch and serving measure the other configs")
    ap.add_argument("--qubos", type=int, default=256)
    ap.add_argument("--jrps", type=int, default=128)
    ap.add_argument("--fp64-stride", type=int, default=1)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--rates", type=float, nargs="+", default=[50, 100, 200, 500, 1000, 2000])
    ap.add_argument("--seconds", type=float, default=2.0)
    ap.add_argument("--pool-qubo", type=int, default=28)
    ap.add_argument("--pool-jrp", type=int, default=12)
    args = ap.parse_args()
    if args.impl == "reference":
        if args.warmup < 3:
            args.warmup = 3
        return run_reference(args)
    if args.workload == "pria":
        return run_pria(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.warmup < 3:
        args.warmup = 3
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
