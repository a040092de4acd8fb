"""Multi-process plumbing: one process per GPU over ``torch.distributed``.

The ray cast shards by frames, views or image tiles with no data-path
collective; the only exchanges are the timing reduction of a benchmark and,
for data-parallel fitting of brick contents, the sum of the texel gradients.
NCCL is used on GPUs, gloo on CPU (tests).  Rendezvous on 127.0.0.1.
"""
from __future__ import annotations

import os
from datetime import timedelta

import torch
import torch.distributed as dist


def env() -> tuple[int, int, int]:
    """(rank, local rank, world size) from the launcher's environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def init(backend: str | None = None, timeout_s: float = 600.0) -> bool:
    """Join the process group when the world has more than one rank."""
    _, _, world = env()
    if world <= 1 or dist.is_initialized():
        return dist.is_initialized()
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    be = backend or ("nccl" if torch.cuda.is_available() else "gloo")
    dist.init_process_group(be, timeout=timedelta(seconds=timeout_s))
    return True


def path_segment(rank: int, world: int, frames: int) -> tuple[int, int]:
    """First frame and frame count of a rank's contiguous share of a path."""
    lo = rank * frames // world
    hi = (rank + 1) * frames // world
    return lo, hi - lo


def views_of_rank(n_views: int, rank: int, world: int) -> list[int]:
    """Round-robin assignment of view indices to ranks."""
    return list(range(rank, n_views, world))


def max_over_ranks(value: float, device: torch.device | str = "cpu") -> float:
    """The largest value over all ranks (device-timed durations)."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_gradients(grad: torch.Tensor) -> torch.Tensor:
    """All-reduce (sum) of a texel-gradient buffer, in place."""
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM)
    return grad


def barrier() -> None:
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def shutdown() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()
