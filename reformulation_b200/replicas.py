"""Multi-GPU runs as independent replicas: one process per GPU, launched by
torchrun (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* in the environment).

PRAQ and PRIA instances are independent, so N GPUs solve N times the work with
no collective on the data path (weak scaling).  torch.distributed carries only
the barrier that brackets a timed region and the max-over-ranks reduction of
its duration: the whole job's rate is the units every rank processed over the
slowest rank's time.

A fixed set of requests (a batch, or a serving stream) is dealt to the GPUs by
`route`: longest-processing-time-first on an estimate of each request's device
work, so that every rank gets about the same bytes to stream; each rank solves
its share alone and `Replicas.gather` brings the results to rank 0 on the host.
"""

from __future__ import annotations

import datetime
import heapq
import os


def work_estimate(instance) -> float:
    """Device bytes one solve of `instance` streams, up to a common factor:
    the per-iteration algorithmic bytes (FP32 iterates) times an iteration
    count that grows slowly with size (PRAQ: n (6R + I) + m (11R + 4I); PRIA:
    15 ND R; iterations ~ 16 log2 of the size, the measured trend of the
    batch workloads).  Only the ratios between requests matter."""
    import math
    if hasattr(instance, "edges"):
        n, m = instance.n, instance.edges
        per_iter = n * 28 + m * 60
        size = n + m
    else:
        nd = instance.entries
        per_iter = 60 * nd
        size = nd
    return per_iter * 16.0 * max(1.0, math.log2(max(size, 2)))


def route(costs, world: int) -> list[list[int]]:
    """Deal items with the given costs to `world` ranks: heaviest first, each
    to the rank with the least total so far (ties to the lower rank).  Every
    item goes to exactly one rank; each rank's list is in the items' order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(s) for s in shares]


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0, device=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            kwargs = {}
            if backend == "nccl" and device is not None:
                kwargs["device_id"] = device
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kwargs)
            self._dist = dist

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, value: float) -> float:
        """The largest `value` over the ranks (every rank gets it)."""
        if self._dist is None:
            return float(value)
        import torch
        dev = self.device if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def gather(self, obj):
        """Every rank's `obj` (picklable) on rank 0, in rank order; None on
        the other ranks.  For host-side results (bounds, iterations, primal
        vectors); on NCCL the pickled bytes pass through a device buffer."""
        if self._dist is None:
            return [obj]
        out = [None] * self.world if self.rank == 0 else None
        self._dist.gather_object(obj, out, dst=0)
        return out

    def whole_job_rate(self, units_per_rank: float, seconds: float) -> float:
        """Units all ranks processed per second of the slowest rank."""
        return self.world * units_per_rank / self.max(seconds)

    def close(self) -> None:
        if self._dist is not None:
            self._dist.barrier()
            self._dist.destroy_process_group()
            self._dist = None
