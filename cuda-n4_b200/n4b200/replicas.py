"""Volume-parallel replicas across GPUs (one process per GPU).

Volumes are independent, so a multi-GPU job shards them across ranks with
no collective on the data path: every rank corrects its own volumes and the
only communication is the timing protocol — a barrier on both sides of the
timed region and the maximum of the per-rank device times.  The process
group is ``torch.distributed`` (NCCL on GPUs; gloo for the CPU tests of this
logic).
"""
from __future__ import annotations

import datetime
import os


def volume_seeds(rank: int, batch: int) -> list:
    """Seeds of the synthetic volumes rank `rank` corrects (disjoint across
    ranks for batch <= 1000)."""
    return [1000 * rank + i for i in range(batch)]


def shard(n: int, rank: int, world: int) -> range:
    """Indices of `n` items owned by `rank`: contiguous, sizes differing by at
    most one."""
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return range(lo, hi)


class Replicas:
    """The timing protocol of a replicated run over an initialised (or
    absent, world 1) process group."""

    def __init__(self, world: int, device=None, backend: str = "nccl", timeout_s: int = 120):
        self.world = world
        self.device = device
        self.dist = None
        if world > 1:
            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    @property
    def rank(self) -> int:
        return self.dist.get_rank() if self.dist is not None else int(os.environ.get("RANK", 0))

    def barrier(self):
        import torch
        if self.dist is not None:
            self.dist.barrier()
        if self.device is not None and self.device.type == "cuda":
            torch.cuda.synchronize(self.device)

    def max_over_ranks(self, x: float) -> float:
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, per_rank_units: int, ms_this_rank: float) -> float:
        """Whole-job units/s: all ranks' units over the slowest rank's time."""
        return self.world * per_rank_units / (self.max_over_ranks(ms_this_rank) / 1000.0)

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
