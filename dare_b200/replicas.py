"""Rank plumbing of multi-GPU runs of the implicit step: one process per GPU,
each an independent replica of the whole workload (the path is not sharded,
so there is no data-path collective).  The only collectives are a barrier
around timed regions and the maximum of the ranks' timings, which makes the
reported time that of the slowest rank.

Ranks come from the launcher's environment (RANK, WORLD_SIZE, LOCAL_RANK,
MASTER_ADDR, MASTER_PORT).  NCCL is the backend on GPUs; gloo runs the same
code on CPU processes.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    @property
    def device(self) -> str:
        """Where reduction operands live: the rank's GPU under NCCL, else the CPU."""
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """The maximum of `x` over all ranks (every rank gets it)."""
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], device=self.device, dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        """Every rank leaves together; call once, after the last collective."""
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
