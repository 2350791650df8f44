"""Process-group plumbing of the multi-GPU modes, one process per GPU.

Ranks from the torchrun environment, barriers, and the maximum (or sum) over ranks of
a rank's device time.  The backend is NCCL on GPUs (the reduction tensor lives on the
rank's device) and gloo on the host (tests).  The data path of a multi-GPU sweep --
the CORE-SG broadcast, the mpts partition and the gather of the trees -- is in
partition.py; replica_throughput is the throughput of independent replicas (every
rank sweeping all K mpts of its own graph).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    """This process's place in the job and the process group (None when alone)."""
    rank: int = 0
    world: int = 1
    local: int = 0
    group: object = None
    device: str = "cpu"

    def barrier(self) -> None:
        if self.group is not None:
            self.group.barrier()

    def max_over_ranks(self, x: float) -> float:
        """max of x over all ranks (every rank gets it); x itself when alone."""
        if self.group is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.group.all_reduce(t, op=self.group.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, x: float) -> float:
        """sum of x over all ranks (every rank gets it); x itself when alone."""
        if self.group is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.group.all_reduce(t, op=self.group.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self.group is not None:
            self.group.destroy_process_group()
            self.group = None


def from_env(backend: str = "nccl", timeout_s: float = 120.0) -> Ranks:
    """Rank, world size and local rank from the torchrun environment (RANK,
    WORLD_SIZE, LOCAL_RANK, MASTER_ADDR/PORT); joins the process group when the world
    has more than one rank.  With NCCL the local rank's GPU becomes the current
    device and the reductions run on it."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    r = Ranks(rank=rank, world=world, local=local)
    if world > 1:
        import torch
        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
            r.device = f"cuda:{local}"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        r.group = dist
    return r


def replica_throughput(world: int, mpts_per_step: int, steps: int, max_total_ms: float) -> float:
    """Whole-job MSTs/s of `world` replicas that each solved `mpts_per_step` MSTs per
    step for `steps` steps, timed by the slowest rank's total device milliseconds."""
    if max_total_ms <= 0:
        raise ValueError("the timed region must be positive")
    return world * mpts_per_step * steps / (max_total_ms / 1000.0)
