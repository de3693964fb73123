"""Independent replicas of the solver, one per process and GPU.

The cavity does not shard (each rank advances its own cavity), so the only
collectives are bookkeeping: a barrier around the timed region and the
maximum of the per-rank times (the slowest rank defines the job's time).
Launched by torchrun; RANK, LOCAL_RANK and WORLD_SIZE come from the
environment, MASTER_ADDR/MASTER_PORT likewise.
"""
from __future__ import annotations

import datetime
import os
from typing import Optional


class Replicas:
    """world == 1: no process group, every call is local."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist

            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, value: float) -> float:
        """Maximum of a float over the ranks (every rank gets it)."""
        if self._dist is None:
            return float(value)
        import torch

        device = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, value: float) -> float:
        if self._dist is None:
            return float(value)
        import torch

        device = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
