"""One frame over several GPUs: one process per GPU (torch.distributed).

Pixels and samples are independent, so a frame shards without any exchange
in the path tracing itself. Two splits:

  by samples (weak scaling: per-GPU work fixed) -- every rank renders the
      whole image with its own range of sample indices (sample_offset =
      rank * spp), so the ranks' samples are disjoint and together are
      world * spp samples per pixel; one sum all-reduce of the HDR image,
      divided by the world size, combines them (`shard_settings`,
      `combine`);
  by rows (strong scaling: the frame fixed) -- rank r renders the band of
      rows `row_band(height, r, world)` of the same image with
      pgpu_render_window, every pixel exactly as a one-GPU render makes it,
      and one all-gather assembles the frame (`gather_rows`). This is the
      fixed-frame form of Pencil's tile farm, whose workers render 64x64
      tiles of one frame (src/distributed.hpp:642-718).

The adjoint shards by samples like the image: each rank differentiates the
loss over its own samples and one sum all-reduce of the FP64 gradient
vectors, divided by the world size, gives the gradient of the combined
image (`combine_gradients`). Batches of scenes shard by scene and need no
exchange at all (`shard_jobs`). NCCL over NVLink on GPUs, gloo on CPU.
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


def row_band(height: int, rank: int, world: int) -> tuple[int, int]:
    """Rows [y0, y1) of a `height`-row image for `rank`: contiguous bands
    whose heights differ by at most one row, in rank order."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(height, world)
    y0 = rank * base + min(rank, extra)
    return y0, y0 + base + (1 if rank < extra else 0)


def gather_rows(band, height: int, world: int, group=None):
    """The full image (height, W, 3) from every rank's band of rows
    (row_band order), on every rank: one all-gather of equal-size buffers
    (bands padded to the tallest)."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return band
    tallest = row_band(height, 0, world)[1]
    pad = torch.zeros((tallest,) + tuple(band.shape[1:]), dtype=band.dtype, device=band.device)
    pad[:band.shape[0]] = band
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    rows = []
    for r in range(world):
        y0, y1 = row_band(height, r, world)
        rows.append(parts[r][:y1 - y0])
    return torch.cat(rows, 0)


def combine_gradients(grads, world: int, group=None):
    """In place: the mean over ranks of each FP64 gradient tensor (the
    gradient of the mean of the ranks' images), with one all-reduce over
    the concatenation of all of them."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return grads
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    flat.div_(world)
    off = 0
    for g in grads:
        n = g.numel()
        g.copy_(flat[off:off + n].view_as(g))
        off += n
    return grads
