"""Failure detection, injected on the host: every case ends in a status code
(and a message), never in a device trap or a hang, and the context keeps
rendering correctly afterwards.

The reference's only failure handling is its distributed mode's socket
timeouts and dead-worker handling (src/distributed.hpp:527-545, 680-684).
Here the faults are corrupt or truncated scene tables (rejected at upload,
before any kernel sees them), a shadow-record store too small for the scene
(PGPU_INJECT_SHADOW_RECORDS: shade stores no record beyond its room and
reports the overflow) and a wall-clock budget smaller than the render
(pgpu_set_timeout: the call returns PGPU_ERR_TIMEOUT while the kernels,
which never wait on anything, run to their end).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import load_golden
from pencil_b200 import _abi as A
from pencil_b200 import workloads as W
from pencil_b200.renderer import RenderSettings
from pencil_b200.scene import Light, Material, Scene

pytestmark = pytest.mark.gpu


def small_scene() -> Scene:
    s = Scene()
    m = s.add_material(Material.diffuse((0.6, 0.5, 0.4)))
    g = s.add_material(Material.dielectric(1.5))
    s.add_sphere((0, 0, 0), 1.0, m)
    s.add_sphere((1.5, 0.2, -0.5), 0.5, g)
    s.add_plane((0, -1, 0), (0, 1, 0), m)
    s.add_light(Light.point((3, 5, -4), (1, 1, 1), 0.3))
    s.add_light(Light.directional((0.2, -1, 0.3), (0.3, 0.3, 0.3)))
    return s


ST = RenderSettings(width=48, height=32, samples=2, pathtrace=True, pathtrace_bounces=5)


def expect(code, fn, *args, match: str | None = None):
    with pytest.raises(A.GpuError) as e:
        fn(*args)
    assert e.value.code == code, str(e.value)
    if match:
        assert match in str(e.value)


def test_corrupt_scene_tables_are_rejected_at_upload(gpu):
    ref_scene = small_scene()
    sid = gpu.upload(ref_scene)
    good = gpu.render(sid, ST)
    # material index out of range
    s = small_scene()
    s.add_sphere((0, 2, 0), 0.5, 7)
    expect(A.ERR_INVALID_ARG, gpu.upload, s, match="material")
    # a NaN primitive parameter
    s = small_scene()
    s.add_sphere((0, float("nan"), 0), 0.5, 0)
    expect(A.ERR_INVALID_ARG, gpu.upload, s, match="non-finite")
    # an infinite radius
    s = small_scene()
    s.add_sphere((0, 0, 3), float("inf"), 0)
    expect(A.ERR_INVALID_ARG, gpu.upload, s, match="non-finite")
    # mesh: indices past the end of a truncated vertex array
    s = small_scene()
    v = np.array([[0, 0, 2], [1, 0, 2], [0, 1, 2], [1, 1, 2]], np.float32)
    s.set_mesh(v[:3], np.array([[0, 1, 2], [1, 3, 2]], np.int32), 0)
    expect(A.ERR_INVALID_ARG, gpu.upload, s, match="out of range")
    # mesh: negative index, material out of range, NaN vertex
    s = small_scene()
    s.set_mesh(v, np.array([[0, -1, 2]], np.int32), 0)
    expect(A.ERR_INVALID_ARG, gpu.upload, s, match="out of range")
    s = small_scene()
    s.set_mesh(v, np.array([[0, 1, 2]], np.int32), 9)
    expect(A.ERR_INVALID_ARG, gpu.upload, s, match="material")
    s = small_scene()
    v2 = v.copy()
    v2[1, 0] = np.nan
    s.set_mesh(v2, np.array([[0, 1, 2]], np.int32), 0)
    expect(A.ERR_INVALID_ARG, gpu.upload, s, match="not finite")
    # the context still renders the good scene, bit for bit
    assert np.array_equal(gpu.render(sid, ST).view(np.uint32), good.view(np.uint32))
    gpu.free(sid)


def test_corrupt_bvh_tables_are_rejected_at_upload(gpu):
    s = small_scene()
    nodes, _ = s.build_bvh()
    leaves = np.nonzero(nodes["left"] < 0)[0]
    bad = nodes.copy()
    bad["right"][leaves[0]] = 99                # leaf primitive out of range
    expect(A.ERR_BVH_INVALID, gpu.upload, s, bad)
    bad = nodes.copy()
    bad["right"][leaves[1]] = bad["right"][leaves[0]]   # a primitive in two leaves
    expect(A.ERR_BVH_INVALID, gpu.upload, s, bad)
    bad = nodes.copy()
    bad["bmin"][0, 1] = np.nan                  # a non-finite box
    expect(A.ERR_BVH_INVALID, gpu.upload, s, bad)
    expect(A.ERR_BVH_INVALID, gpu.upload, s, nodes[:-1])   # truncated table
    sid = gpu.upload(s, nodes)
    assert np.isfinite(gpu.render(sid, ST)).all()
    gpu.free(sid)


@pytest.mark.parametrize("pathtrace", [True, False])
def test_shadow_record_overflow_is_reported(gpu, monkeypatch, pathtrace):
    """The scene needs two shadow records per path-trace vertex (two lights;
    Whitted: 4 soft samples + 1); the store is cut to one."""
    s = small_scene()
    sid = gpu.upload(s)
    st = dataclasses.replace(ST, pathtrace=pathtrace, engine=A.ENGINE_WAVEFRONT)
    good = gpu.render(sid, st)
    monkeypatch.setenv("PGPU_INJECT_SHADOW_RECORDS", "1")
    expect(A.ERR_QUEUE_OVERFLOW, gpu.render, sid, st, match="overflow")
    expect(A.ERR_QUEUE_OVERFLOW, gpu.render_batch, [sid, sid], [st, st], match="overflow")
    monkeypatch.delenv("PGPU_INJECT_SHADOW_RECORDS")
    assert np.array_equal(gpu.render(sid, st).view(np.uint32), good.view(np.uint32))
    gpu.free(sid)


def test_time_budget_returns_timeout_and_context_recovers(gpu):
    """The full benchmark frame (about 25 ms of device work) against a 1 ms
    budget: PGPU_ERR_TIMEOUT, for a single render, a batch and an adjoint;
    then, without a budget, the same context renders the frame exactly as a
    render that never timed out."""
    w = W.sphere_cloud()
    sid = gpu.upload(w.scene)
    st = dataclasses.replace(w.settings, engine=A.ENGINE_WAVEFRONT)
    ref = gpu.render(sid, st)
    gpu.set_timeout(1)
    try:
        expect(A.ERR_TIMEOUT, gpu.render, sid, st, match="budget")
        expect(A.ERR_TIMEOUT, gpu.render_batch, [sid, sid], [st, st], match="budget")
        dl = np.ones((st.height, st.width, 3), np.float32)
        expect(A.ERR_TIMEOUT, gpu.adjoint, sid, st, dl, w.scene.n_materials,
               len(w.scene.lights), match="budget")
        # a budget the work fits in
        gpu.set_timeout(60_000)
        assert np.array_equal(gpu.render(sid, st).view(np.uint32), ref.view(np.uint32))
    finally:
        gpu.set_timeout(0)
    assert np.array_equal(gpu.render(sid, st).view(np.uint32), ref.view(np.uint32))
    expect(A.ERR_INVALID_ARG, gpu.set_timeout, -5)
    gpu.free(sid)


def test_invalid_launch_shapes_are_rejected(gpu):
    scene, fx = load_golden("c1")
    sid = gpu.upload(scene, fx["nodes"])
    for bs in (32, 100, 512, -1):
        expect(A.ERR_INVALID_ARG, gpu.render, sid, dataclasses.replace(ST, block_size=bs),
               match="block_size")
    expect(A.ERR_INVALID_ARG, gpu.render, sid, dataclasses.replace(ST, refill_below=40))
    for q in (-1, (1 << 28) + 1):
        expect(A.ERR_INVALID_ARG, gpu.render, sid, dataclasses.replace(ST, queue_capacity=q),
               match="queue_capacity")
    for bs in (64, 128, 256):          # every supported shape gives the same image
        a = gpu.render(sid, dataclasses.replace(ST, block_size=bs, sort_key=3))
        assert np.array_equal(a.view(np.uint32), gpu.render(sid, ST).view(np.uint32))
    gpu.free(sid)
