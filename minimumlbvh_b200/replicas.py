"""Multi-GPU plumbing of the benchmark: one process per GPU, each running its
own replica of the workload (the build and the traversal of one frame do not
shard: the build is a global sort and a bottom-up climb, and the rays of a
frame fit one GPU). No data crosses ranks; the process group only aligns the
start and end of timed regions and takes the maximum of the per-rank times.

`Replicas` reads RANK / WORLD_SIZE / LOCAL_RANK from the environment
(torchrun); with one process it is a no-op.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0, device=None):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local_rank = int(os.environ.get("LOCAL_RANK", 0))
        self.device = device
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """The maximum of x over all ranks (every rank must call it)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    @property
    def is_root(self) -> bool:
        return self.rank == 0

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
