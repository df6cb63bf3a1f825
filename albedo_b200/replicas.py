"""Replica runs on several GPUs of one node.

A pixel's samples run in sequence on its own random stream (the reference's
renderPixel loop, render/render_image.cpp:27-44), so a render does not shard
across GPUs without changing results. Several GPUs therefore each render their
own copy of the workload: there is no collective on the data path, and the
whole job's throughput is every rank's work over the slowest rank's time.
"""

from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Ranks:
    rank: int
    world: int
    local_rank: int


def ranks_from_env() -> Ranks:
    """RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them (one process without them)."""
    return Ranks(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The largest `value` over all ranks of an initialized process group (the
    value itself without one). `device` is where the reduction runs: "cuda" for
    NCCL, "cpu" for gloo."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_throughput(units_per_rank_step: float, steps: int, world: int, slowest_seconds: float) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    if slowest_seconds <= 0:
        raise ValueError("the timed region must take some time")
    return world * units_per_rank_step * steps / slowest_seconds
