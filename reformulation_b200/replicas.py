"""Multi-GPU runs as independent replicas: one process per GPU, launched by
torchrun (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* in the environment).

PRAQ and PRIA instances are independent, so N GPUs solve N times the work with
no collective on the data path (weak scaling).  torch.distributed carries only
the barrier that brackets a timed region and the max-over-ranks reduction of
its duration: the whole job's rate is the units every rank processed over the
slowest rank's time.
"""

from __future__ import annotations

import datetime
import os


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

    def whole_job_rate(self, units_per_rank: float, seconds: float) -> float:
        """Units all ranks processed per second of the slowest rank."""
        return self.world * units_per_rank / self.max(seconds)

    def close(self) -> None:
        if self._dist is not None:
            self._dist.barrier()
            self._dist.destroy_process_group()
            self._dist = None
