"""The multi-GPU path of bench.py is N independent replicas: a barrier and a
max-over-ranks reduction of the timed region, no collective on the data
path.  Checked here with two gloo ranks on the CPU (the same calls the NCCL
ranks make on GPUs): every rank sees the slowest rank's time, and the whole
job's rate is the units of all ranks over that time."""

import multiprocessing as mp
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from reformulation_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    rep.barrier()
    seconds = 1.0 + rank            # rank 1 is the slower one
    out.put((rank, rep.max(seconds), rep.whole_job_rate(10, seconds), rep.world))
    rep.close()


def test_two_gloo_replicas_reduce_to_the_slowest():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, rate, world in got:
        assert world == 2 and slowest == 2.0
        assert rate == pytest.approx(2 * 10 / 2.0)


def test_single_process_needs_no_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    from reformulation_b200.replicas import Replicas
    rep = Replicas("gloo")
    assert rep.world == 1 and rep.max(3.5) == 3.5 and rep.whole_job_rate(4, 2.0) == 2.0
    rep.barrier()
    rep.close()
