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


def test_row_bands_partition_the_frame():
    from pencil_b200.distributed import row_band
    for h in (1, 7, 720):
        for world in (1, 2, 3, 8):
            if world > h:
                continue
            bands = [row_band(h, r, world) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == h
            assert all(a[1] == b[0] for a, b in zip(bands, bands[1:]))
            sizes = [b - a for a, b in bands]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        row_band(10, 3, 3)


def _strong_rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    """Fixed frame: this rank renders its band of rows (a window of the
    image) and the all-gather assembles the frame; then the adjoint of its
    own samples and the gradient all-reduce."""
    import torch.distributed as dist
    from oracle import oracle as O
    from pencil_b200 import workloads as W
    from pencil_b200.distributed import combine_gradients, gather_rows, row_band
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = W.three_spheres_pt(width=24, height=19, samples=2, depth=3)
    y0, y1 = row_band(w.settings.height, rank, world)
    band, _, _ = O.Oracle(w.scene).render_split(
        w.settings, threads=1, window=(0, y0, w.settings.width, y1 - y0))
    frame = gather_rows(torch.from_numpy(np.ascontiguousarray(band)), w.settings.height, world)
    np.save(os.path.join(out_dir, f"frame{rank}.npy"), frame.numpy())
    wa, _, _ = W.adjoint_box(20, 16, 16, 2, 3, seed=3)
    dl = np.random.default_rng(5).normal(size=(16, 16, 3)).astype(np.float32)
    da, de, dli, _ = O.Oracle(wa.scene).adjoint(shard_settings(wa.settings, rank, world), dl,
                                                threads=1)
    grads = [torch.from_numpy(np.ascontiguousarray(g)) for g in (da, de, dli)]
    combine_gradients(grads, world)
    np.savez(os.path.join(out_dir, f"grad{rank}.npz"), *[g.numpy() for g in grads])
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_fixed_frame_rows_and_gradient_all_reduce(tmp_path):
    """Strong scaling: the frame assembled from two ranks' row bands equals
    the one-process render bit for bit; the all-reduced FP64 gradients equal
    the mean of the two ranks' gradients computed here."""
    import socket

    import torch.multiprocessing as mp
    from oracle import oracle as O
    from pencil_b200 import workloads as W
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    mp.start_processes(_strong_rank_main, args=(world, port, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    w = W.three_spheres_pt(width=24, height=19, samples=2, depth=3)
    full, _, _ = O.Oracle(w.scene).render_split(w.settings, threads=1)
    wa, _, _ = W.adjoint_box(20, 16, 16, 2, 3, seed=3)
    dl = np.random.default_rng(5).normal(size=(16, 16, 3)).astype(np.float32)
    per_rank = [O.Oracle(wa.scene).adjoint(shard_settings(wa.settings, r, world), dl, threads=1)
                for r in range(world)]
    for r in range(world):
        frame = np.load(tmp_path / f"frame{r}.npy")
        assert np.array_equal(frame.view(np.uint32), full.view(np.uint32))
        with np.load(tmp_path / f"grad{r}.npz") as z:
            got = [z[f"arr_{k}"] for k in range(3)]
        for k in range(3):
            want = (per_rank[0][k] + per_rank[1][k]) / 2
            assert np.allclose(got[k], want, rtol=1e-12, atol=1e-15)
    assert not np.array_equal(per_rank[0][0], per_rank[1][0])
