"""Replica bookkeeping for runs with one independent box per GPU (no data-path collective).

The time-step path does not shard (one box needs a global transpose per 3-D
transform), so N GPUs run N independent boxes.  The whole-job rate is
N*steps / (max over ranks of the device time); the collective is used only
for that maximum and for barriers.
"""
from __future__ import annotations


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, steps: int, max_seconds: float) -> float:
    """Steps per second of the whole job (all replicas)."""
    return world * steps / max_seconds
