"""Independent replicas of one run on N GPUs of a node (one process per GPU).

A single vortex ring at the benchmark sizes fits one B200, and the RK3 core
has no exchange between replicas, so N > 1 means N independent runs; the only
collectives are the barrier around the timed region and the max-over-ranks
of the device-timed duration (the job's time is its slowest rank's).

The process group is NCCL on GPUs (the launcher sets RANK, WORLD_SIZE,
LOCAL_RANK, MASTER_ADDR and MASTER_PORT) and gloo for the CPU tests.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Replicas:
    rank: int
    world: int
    local: int
    backend: str | None  # None: single process, no process group

    @property
    def distributed(self) -> bool:
        return self.backend is not None

    def barrier(self) -> None:
        if self.distributed:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        """Largest x over the ranks (every rank gets it)."""
        if not self.distributed:
            return float(x)
        import torch
        import torch.distributed as dist
        dev = torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.distributed:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
            self.backend = None


def init(backend: str = "nccl", timeout_s: float = 300.0) -> Replicas:
    """Join the launcher's process group when WORLD_SIZE > 1."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return Replicas(rank, world, local, None)
    import torch
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, **kw)
    return Replicas(rank, world, local, backend)


def throughput(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job rate: the units all ranks processed over the slowest rank's time."""
    return world * units_per_rank / seconds_max
