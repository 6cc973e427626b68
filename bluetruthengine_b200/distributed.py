"""Multi-GPU rendering: one process per GPU, samples sharded by index.

Camera paths are independent, so N ranks render the same view with disjoint
sample indices (the RNG seed is hashUint(pixel ^ sample*0x9e3779b9), so every
rank draws different, reproducible streams).  The only exchange is the final
sum of the FP64 per-pixel accumulators, one all-reduce of W*H*3 doubles
(NCCL over NVLink on GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def sample_base(rank: int, frames: int, samples_per_frame: int) -> int:
    """First sample index of `rank` when every rank renders `frames` frames of
    `samples_per_frame` paths per pixel: rank r owns [r*F*S, (r+1)*F*S)."""
    return rank * frames * samples_per_frame


def merge_accumulators(sum_f64, samples_this_rank: int, group=None):
    """All-reduce the per-pixel FP64 sums and sample counts; returns the mean image
    (float64) identical on every rank.  `sum_f64` is a torch tensor or numpy array.

    Wavefront mode: `samples_this_rank` is the rank's samples per pixel.  In megakernel mode the
    accumulator is a sum of per-frame means, so pass the rank's frame count instead."""
    import torch
    import torch.distributed as dist
    t = sum_f64 if isinstance(sum_f64, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(sum_f64))
    t = t.to(torch.float64)
    n = torch.tensor([float(samples_this_rank)], dtype=torch.float64, device=t.device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
    return t / n


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The slowest rank's time (the job's time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
