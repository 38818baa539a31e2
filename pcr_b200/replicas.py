"""Multi-GPU replicas: one process per GPU, each rendering its own seeded
batch with no data-path collective (requests are independent, so the work
shards without an exchange).  The only collectives are the ones the timing
needs: a barrier around the timed region and max / sum reductions of
per-rank scalars (time is the max over ranks, work the sum).

The launcher (torchrun) sets RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR /
MASTER_PORT.  `bench.py` uses the "nccl" backend on GPUs; the CPU tests run
the same code with "gloo".
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: int = 300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
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

    def seed(self, base: int) -> int:
        """Each replica renders its own batch (weak scaling)."""
        return base + self.rank

    def _tensor(self, x: float):
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self) -> None:
        if self.backend == "nccl":
            import torch
            torch.cuda.synchronize()
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.dist:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
