"""Autotuner of the wavefront engine's launch parameters.

The wavefront renderer has four knobs whose best values depend on the
workload (image size, samples, scene, light count) and the GPU:

  queue_capacity  paths in flight per chunk: more paths keep late bounces
                  busy but cost scratch memory (about 212 B per path plus
                  64 B per shadow record a vertex can make); candidates
                  from 2^20 to 2^26 paths, as far as half the free device
                  memory holds them
  refill_below    a warp of the persistent traversal kernels fetches new rays
                  once at most this many of its lanes are still traversing
  sort_key        0: queue order; 1: rays binned by direction octant;
                  2: shadow work sorted by origin cell and octant; 3: also the
                  extension rays after the first bounce
  block_size      threads per block of the wavefront kernels (64, 128, 256):
                  the launch shape, which sets how many warps of a block
                  share its scheduling and its shared-memory stacks

`autotune` times candidates with short device-resident renders (CUDA events
on the render stream, a warm-up render first) by coordinate search: capacity
first, then the refill threshold, the sort key and the block size. Results
are cached in a JSON file keyed by the workload's shape, so a renderer pays
the search once.
"""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

import numpy as np

from . import _abi as A
from .renderer import GpuContext, RenderSettings

CACHE = Path(os.environ.get("PGPU_AUTOTUNE_CACHE",
                            Path.home() / ".cache" / "pencil_b200" / "autotune.json"))

CAPACITIES = (1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25, 1 << 26)
# scratch per path in flight, bounded above: path state 128 B, queues 64 B,
# sort lists 20 B and up to four 64-byte shadow records
SCRATCH_BYTES_PER_PATH = 512
REFILLS = (12, 16, 20, 24)
SORT_KEYS = (0, 1, 2, 3)
BLOCKS = (64, 128, 256)


def signature(scene, settings_list: list[RenderSettings]) -> str:
    """Shape of a (batched) workload: scene sizes, light setup, image sizes,
    samples and depth."""
    h = hashlib.sha256()
    h.update(np.array([scene.n_unified, scene.n_materials, len(scene.lights)], np.int64).tobytes())
    for st in settings_list:
        h.update(np.array([st.width, st.height, st.samples, st.pathtrace_bounces,
                           st.max_depth, int(st.pathtrace)], np.int64).tobytes())
    return h.hexdigest()[:24]


def _time_device(ctx: GpuContext, render, reps: int) -> float:
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream)
    render()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        render()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(ctx: GpuContext, sids: list[int], settings: list[RenderSettings], scene=None,
             reps: int = 2, use_cache: bool = True, log=None) -> dict:
    """Pick queue_capacity / refill_below / sort_key / block_size for
    rendering `sids` with `settings` (one job: a single render; several: one
    batch). Returns {"queue_capacity", "refill_below", "sort_key",
    "block_size", "ms", "trials"} and applies the choice to every settings
    object."""
    import torch
    key = signature(scene, settings) if scene is not None else None
    cache = {}
    if use_cache and key and CACHE.exists():
        try:
            cache = json.loads(CACHE.read_text())
        except (OSError, ValueError):
            cache = {}
        if key in cache and "block_size" in cache[key]:
            best = cache[key]
            for st in settings:
                st.queue_capacity, st.refill_below = best["queue_capacity"], best["refill_below"]
                st.sort_key, st.block_size = best["sort_key"], best["block_size"]
            return dict(best, cached=True)
    outs = [torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
            for st in settings]
    total_paths = sum(st.width * st.height * st.samples ** 2 for st in settings)

    def render():
        if len(sids) == 1:
            ctx.render_device(sids[0], settings[0], outs[0].data_ptr())
        else:
            ctx.render_batch(sids, settings, device_ptrs=[o.data_ptr() for o in outs])

    def apply(q, r, s, b):
        for st in settings:
            st.engine = A.ENGINE_WAVEFRONT
            st.queue_capacity, st.refill_below, st.sort_key, st.block_size = q, r, s, b

    trials = []

    def trial(q, r, s, b):
        apply(q, r, s, b)
        ms = _time_device(ctx, render, reps)
        trials.append({"queue_capacity": q, "refill_below": r, "sort_key": s, "block_size": b,
                       "ms": ms})
        if log:
            log(f"autotune q={q} refill={r} sort={s} block={b}: {ms:.2f} ms")
        return ms

    # capacities whose scratch fits in half the free device memory
    room = torch.cuda.mem_get_info()[0] // 2 // SCRATCH_BYTES_PER_PATH
    fit = [q for q in CAPACITIES if q <= room] or [CAPACITIES[0]]
    caps = [q for q in fit if q < total_paths] + [min(total_paths, fit[-1])]
    caps = sorted(set(caps))
    q_best = min(caps, key=lambda q: trial(q, 20, 0, 128))
    r_best = min(REFILLS, key=lambda r: trial(q_best, r, 0, 128))
    s_best = min(SORT_KEYS, key=lambda s: trial(q_best, r_best, s, 128))
    b_best = min(BLOCKS, key=lambda b: trial(q_best, r_best, s_best, b))
    best_ms = min(t["ms"] for t in trials if t["queue_capacity"] == q_best and
                  t["refill_below"] == r_best and t["sort_key"] == s_best and
                  t["block_size"] == b_best)
    best = {"queue_capacity": q_best, "refill_below": r_best, "sort_key": s_best,
            "block_size": b_best, "ms": best_ms}
    apply(q_best, r_best, s_best, b_best)
    if use_cache and key:
        cache[key] = best
        try:
            CACHE.parent.mkdir(parents=True, exist_ok=True)
            CACHE.write_text(json.dumps(cache))
        except OSError:
            pass
    return dict(best, trials=trials, cached=False)
