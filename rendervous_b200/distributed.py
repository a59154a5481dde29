"""Data-parallel rendering across ranks (one process per GPU).

Pixels and paths are independent, so every rank renders the whole image with
its own Philox key and the ranks sum their gradients -- the step of a
data-parallel inverse-rendering loop.  Timing follows the slowest rank.
These helpers are what bench.py runs under torchrun (backend nccl); the
tests run them on CPU ranks (backend gloo).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def rank_seed(step: int, rank: int) -> int:
    """Philox key of `rank`'s paths at `step`: the rank in the key's high 32-bit
    word and the step in the low one, so two (rank, step) pairs share a key only
    if both are equal (steps below 2^32, ranks below 2^31)."""
    if not (0 <= step < (1 << 32)) or not (0 <= rank < (1 << 31)):
        raise ValueError(f"rank_seed: step {step} or rank {rank} out of range")
    return ((rank + 1) << 32) | step


def allreduce_grads(params) -> None:
    """Sums the .grad of every parameter over the ranks (in place)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return
    for p in params:
        if p.grad is not None:
            dist.all_reduce(p.grad)


def _reduce(value: float, op, device) -> float:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over the ranks (a time: the job ends with its slowest rank)."""
    return _reduce(value, dist.ReduceOp.MAX if dist.is_available() else None, device)


def sum_over_ranks(value: float, device=None) -> float:
    """The sum over the ranks (work done by the whole job)."""
    return _reduce(value, dist.ReduceOp.SUM if dist.is_available() else None, device)
