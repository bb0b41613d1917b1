"""Weak-scaling replicas across ranks (one process per GPU).

The trace shards by rays with no data-path exchange: each rank traces its
own seeded beam through its own copy of the grid. The only collectives are
the barriers around the timed region and two scalar reductions, the largest
elapsed time over ranks and the total ray-steps, from which the whole-job
throughput is (total ray-steps) / (max time). They run over NCCL between
GPUs and over gloo in the CPU tests.
"""
from __future__ import annotations

import datetime
import os
from typing import Optional, Tuple

import torch


def rank_env() -> Tuple[int, int, int]:
    """(world_size, rank, local_rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's workload: distinct rays (and fields) per rank."""
    return int(seed) + 1000 * int(rank)


def init(world: int, device: Optional[torch.device] = None, backend: str = "nccl", timeout_s: float = 120.0):
    """The process group for world > 1 (None for a single process). A short
    timeout makes a rank that waits on a missing peer end with an error."""
    if world <= 1:
        return None
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl" and device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def job_totals(dist, elapsed_ms: float, ray_steps: float, device) -> Tuple[float, float]:
    """(max elapsed ms over ranks, sum of ray-steps over ranks)."""
    if dist is None:
        return float(elapsed_ms), float(ray_steps)
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    s = torch.tensor([ray_steps], dtype=torch.float64, device=device)
    dist.all_reduce(s)
    return float(t[0]), float(s[0])


def finish(dist) -> None:
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
