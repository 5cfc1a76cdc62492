"""Multi-GPU sharding logic on CPU: world size 2, gloo backend.

The frame shards by sample range (no exchange while tracing) and combines
with one all-reduce; batches shard by scene. The ranks here render with the
oracle's restatement of the GPU estimator on the CPU, so the combined image
can be checked against the same renders made in this process.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from pencil_b200.distributed import sample_range, shard_jobs, shard_settings
from pencil_b200.renderer import RenderSettings

torch = pytest.importorskip("torch")


def test_shards_have_disjoint_samples_covering_the_frame():
    st = RenderSettings(width=8, height=6, samples=2, sample_offset=3)
    for world in (1, 2, 3, 8):
        seen = []
        for r in range(world):
            sh = shard_settings(st, r, world)
            assert (sh.width, sh.height, sh.samples) == (8, 6, 2)
            seen.extend(sample_range(sh))
        assert sorted(seen) == list(range(3, 3 + 4 * world))
    assert st.sample_offset == 3          # the caller's settings are untouched
    with pytest.raises(ValueError):
        shard_settings(st, 2, 2)


def test_batch_shards_partition_the_scenes():
    cost = [5, 1, 9, 3, 3, 7, 2]
    for world in (1, 2, 3):
        parts = [shard_jobs(len(cost), r, world, cost) for r in range(world)]
        assert sorted(j for p in parts for j in p) == list(range(len(cost)))
        loads = [sum(cost[j] for j in p) for p in parts]
        assert max(loads) - min(loads) <= max(cost)
    assert shard_jobs(4, 0, 2) == [0, 2] and shard_jobs(4, 1, 2) == [1, 3]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch.distributed as dist
    from oracle import oracle as O
    from pencil_b200 import workloads as W
    from pencil_b200.distributed import combine
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = W.three_spheres_pt(width=24, height=18, samples=2, depth=3)
    img = O.Oracle(w.scene).render_split(shard_settings(w.settings, rank, world), threads=1)
    img = img[0] if isinstance(img, tuple) else img
    t = torch.from_numpy(np.ascontiguousarray(img))
    combine(t, world)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_combine_to_the_mean_of_their_sample_ranges(tmp_path):
    import socket

    import torch.multiprocessing as mp
    from oracle import oracle as O
    from pencil_b200 import workloads as W
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    got = [np.load(tmp_path / f"rank{r}.npy") for r in range(world)]
    w = W.three_spheres_pt(width=24, height=18, samples=2, depth=3)
    parts = []
    for r in range(world):
        img = O.Oracle(w.scene).render_split(shard_settings(w.settings, r, world), threads=1)
        parts.append((img[0] if isinstance(img, tuple) else img).astype(np.float32))
    want = (parts[0] + parts[1]) / np.float32(2)
    for g in got:
        assert np.allclose(g, want, rtol=1e-6, atol=1e-7)
    assert not np.array_equal(parts[0], parts[1])     # the ranks drew different samples
