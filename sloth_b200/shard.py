"""One job's rays split over the ranks of a process group.

The reference traces every ray of a job in one process (its vmap over rays,
src/core/propagator.py:785-793; it states that it does not shard rays over
devices, :697-699). Rays are independent and the grid is small next to a
GPU's memory, so a job partitions by rays: every rank packs its own copy of
the grid, traces a contiguous slice of the rays, and the per-ray outputs are
all-gathered into ray order on every rank. The only exchange is that gather
(NCCL between GPUs, gloo on the host), plus two scalar reductions: the total
ray-steps and the longest trace time over the ranks.
"""
from __future__ import annotations

from typing import Tuple

import numpy as np
import torch


def group_info(group) -> Tuple[int, int]:
    """(world size, rank) of `group` (torch.distributed)."""
    import torch.distributed as dist
    return dist.get_world_size(group), dist.get_rank(group)


def comm_device(group, device=None) -> torch.device:
    """Where the group's collectives run: the rank's GPU for NCCL, else the host."""
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return device if device is not None else torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def shard_bounds(n: int, world: int, rank: int) -> Tuple[int, int]:
    """[lo, hi) of rank `rank`'s contiguous slice of n rays; the first n % world
    ranks take one ray more, so slices differ by one ray at most."""
    base, extra = divmod(int(n), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_rays(local: np.ndarray, n: int, group, device) -> np.ndarray:
    """Concatenate every rank's slice of a per-ray output (rays on the last
    axis) in rank order, on every rank. Slices are padded to the longest one
    for the all-gather and trimmed after it."""
    import torch.distributed as dist
    world, _ = group_info(group)
    longest = shard_bounds(n, world, 0)[1]
    t = torch.from_numpy(np.ascontiguousarray(local))
    pad = longest - t.shape[-1]
    if pad:
        t = torch.nn.functional.pad(t.reshape(-1, t.shape[-1]), (0, pad)).reshape(*t.shape[:-1], longest)
    t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out = []
    for r, p in enumerate(parts):
        lo, hi = shard_bounds(n, world, r)
        out.append(p[..., : hi - lo].cpu())
    return torch.cat(out, dim=-1).numpy()


def reduce_scalar(value: float, group, device, op: str) -> float:
    """Sum ('sum') or maximum ('max') of a scalar over the group's ranks."""
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX, group=group)
    return float(t[0])
