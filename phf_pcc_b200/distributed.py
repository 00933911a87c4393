"""Grid-point sharding across processes (one per GPU) with a sum of the accumulators.

The projected sums run over independent grid points, so one evaluation can be split across
ranks: rank r evaluates a contiguous block of the flattened points (the split the reference
computes at PHF_fort/PHFTools.f90:53-57 and leaves disabled at :85-86), and the H, S, Yg, Yr
slot sums are added with one all-reduce -- the only collective (2 nci^2 (1 + M N) complex
numbers per evaluation).  Independent instances need no collective at all.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

__all__ = ["point_range", "allreduce_accumulators", "ShardedPlan"]


def point_range(npoints: int, rank: int, world: int):
    """Contiguous block [begin, end) of ``npoints`` for ``rank``; the first npoints % world
    ranks get one extra point."""
    base, extra = divmod(int(npoints), int(world))
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def allreduce_accumulators(tensors, group=None):
    """Sum complex accumulators over the ranks of ``group`` in place (as real views)."""
    for t in tensors:
        dist.all_reduce(torch.view_as_real(t), op=dist.ReduceOp.SUM, group=group)
    return tensors


class ShardedPlan:
    """A plan over this rank's block of grid points whose ``eval_device`` returns the full sums."""

    def __init__(self, npoints: int, group=None, **plan_kwargs):
        from .api import Plan

        self.group = group
        rank = dist.get_rank(group) if dist.is_initialized() else 0
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.range = point_range(npoints, rank, world)
        self.plan = Plan(point_range=self.range, **plan_kwargs)
        self.nci, self.gradient, self._g = self.plan.nci, self.plan.gradient, self.plan._g

    def eval_device(self, C, out=None, stream=None):
        hs, yg, yr = self.plan.eval_device(C, out=out, stream=stream)
        if dist.is_initialized() and dist.get_world_size(self.group) > 1:
            allreduce_accumulators((hs, yg, yr), self.group)
        return hs, yg, yr

    def close(self):
        self.plan.close()
