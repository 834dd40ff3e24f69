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


def test_route_deals_every_item_once_and_balances():
    from reformulation_b200.replicas import route
    costs = [5, 1, 9, 3, 3, 7, 2, 8, 1, 6]
    for world in (1, 2, 3, 8, 12):
        shares = route(costs, world)
        assert len(shares) == world
        flat = sorted(k for s in shares for k in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[k] for k in s) for s in shares]
        # LPT: no rank above the average by more than the largest item
        assert max(loads) <= sum(costs) / world + max(costs)
    assert route([], 3) == [[], [], []]


def test_work_estimate_orders_by_size():
    from reformulation_b200.instances import jrp_demand, qubo_uniform_edges
    from reformulation_b200.replicas import work_estimate
    small, big = qubo_uniform_edges(1, 500, 2000), qubo_uniform_edges(1, 5000, 40000)
    assert work_estimate(big) > work_estimate(small) > 0
    assert work_estimate(jrp_demand(1, 20, 100)) > work_estimate(jrp_demand(1, 5, 30))


def _routed_rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from reformulation_b200.replicas import Replicas, route
    rep = Replicas("gloo", timeout_s=60)
    requests = [(rid, 1 + (rid * 7) % 11) for rid in range(23)]      # (id, cost)
    mine = route([c for _, c in requests], rep.world)[rep.rank]
    # the engine, mocked: a request's result is its id and the rank that ran it
    results = [(requests[k][0], rep.rank) for k in mine]
    gathered = rep.gather(results)
    if rep.rank == 0:
        out.put(gathered)
    rep.close()


def test_two_gloo_ranks_route_and_gather():
    """A request list routed over two ranks (engine mocked on the CPU): each
    rank solves only its share, and rank 0 gathers every request exactly
    once."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_routed_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert len(gathered) == 2
    done = [rid for part in gathered for rid, _ in part]
    assert sorted(done) == list(range(23))
    assert {r for _, r in gathered[0]} == {0} and {r for _, r in gathered[1]} == {1}
    assert gathered[0] and gathered[1]
