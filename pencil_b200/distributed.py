"""One frame over several GPUs: one process per GPU (torch.distributed).

Pixels and samples are independent, so the frame shards without any
exchange in the path tracing itself: every rank renders the whole image
with its own range of sample indices (sample_offset = rank * spp), so the
ranks' samples are disjoint and together are world * spp samples per pixel.
The one exchange is combining the images: a sum all-reduce of the HDR image
divided by the world size (NCCL over NVLink on GPUs, gloo on CPU). Batches
of scenes shard by scene and need no exchange at all.
"""
from __future__ import annotations

import dataclasses

from .renderer import RenderSettings


def shard_settings(settings: RenderSettings, rank: int, world: int) -> RenderSettings:
    """This rank's copy of `settings`: the same image, sample indices
    [offset + rank * spp, offset + (rank + 1) * spp)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    spp = settings.samples * settings.samples
    return dataclasses.replace(settings, sample_offset=settings.sample_offset + rank * spp)


def sample_range(settings: RenderSettings) -> range:
    """Sample indices a render with `settings` draws for every pixel."""
    spp = settings.samples * settings.samples
    return range(settings.sample_offset, settings.sample_offset + spp)


def combine(image, world: int, group=None):
    """In place: the mean of the ranks' images (every rank gets it)."""
    import torch.distributed as dist
    if world > 1:
        dist.all_reduce(image, op=dist.ReduceOp.SUM, group=group)
        image.div_(world)
    return image


def shard_jobs(n_jobs: int, rank: int, world: int, cost=None) -> list[int]:
    """Scenes of a batch for this rank: greedy balance of `cost` (paths per
    scene; equal when omitted), largest first, ties to the lower rank.
    Every scene goes to exactly one rank."""
    costs = list(cost) if cost is not None else [1] * n_jobs
    if len(costs) != n_jobs:
        raise ValueError("one cost per job")
    load = [0] * world
    mine: list[int] = []
    for j in sorted(range(n_jobs), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += costs[j]
        if r == rank:
            mine.append(j)
    return sorted(mine)
