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

    def sum_array(self, a):
        """Element-wise sum of a numpy array over the ranks (all ranks get it)."""
        import numpy as np
        if not self.dist:
            return np.asarray(a)
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def close(self) -> None:
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def sample_range(spp: int, rank: int, world: int):
    """Rank's contiguous share [begin, end) of the samples 0..spp-1."""
    base, extra = divmod(spp, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def split_render(ctx, sid: int, desc, rep: Replicas):
    """One render split across the replicas by sample range (the multi-GPU
    single render): every path's random numbers depend on its pixel and
    sample number only, so each rank traces its own samples of every aa
    round; the partial HDR images (each divided by the full samples * aa)
    are summed by an all-reduce and tone-mapped on the device.  Returns
    (hdr, rgb8) on every rank."""
    import copy

    import numpy as np
    b, e = sample_range(desc.samples, rep.rank, rep.world)
    if e > b:
        d = copy.copy(desc)
        d.sample_begin, d.sample_end = b, e
        part = ctx.render(sid, d, want_rgb=False)[0]
    else:
        part = np.zeros((desc.height, desc.width, 3), np.float32)
    hdr = rep.sum_array(part).astype(np.float32)
    return hdr, ctx.tonemap(hdr, aces=bool(desc.aces), denoise=bool(desc.denoise))
