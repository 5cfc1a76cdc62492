"""pgpu_set_traversal_tree: the wide traversals walk a tree built on the
device over the uploaded tree's leaves -- a linear BVH, or a binned SAH tree
over centroid bounds on three axes -- instead of the uploaded tree.

The leaves keep the uploaded tree's boxes and slots (its DFS leaf order,
which decides among hits at equal distance as BVHNode::hit does,
src/bvh.hpp:31-37), so hit distances must be bit-identical and the hit
primitives and rendered pixels equal but where rounding at a box face makes
the order of the walk matter (the same bound the wavefront and the
megakernel are held to on Pencil's own tree). Both engines walk the tree
chosen; the binary tree the upload keeps stays the uploaded one."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN_SCENES, load_golden
from pencil_b200 import _abi as A
from pencil_b200 import workloads as W
from pencil_b200.renderer import RenderSettings

pytestmark = pytest.mark.gpu


MODES = [A.TRAVERSAL_LBVH, A.TRAVERSAL_SAH]


def upload_both(gpu, scene, nodes=None, mode=A.TRAVERSAL_LBVH):
    """The scene uploaded twice: on the uploaded tree and on a device tree."""
    a = gpu.upload(scene, nodes)
    gpu.set_traversal_tree(mode)
    try:
        b = gpu.upload(scene, nodes)
    finally:
        gpu.set_traversal_tree(A.TRAVERSAL_UPLOADED)
    return a, b


def same_pixels(x, y) -> float:
    return float(np.all(x.view(np.uint32) == y.view(np.uint32), axis=2).mean())


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", GOLDEN_SCENES)
def test_device_traversal_tree_finds_the_same_hits(gpu, name, mode):
    scene, fx = load_golden(name)
    a, b = upload_both(gpu, scene, fx["nodes"], mode)
    ia, ib = gpu.scene_info(a), gpu.scene_info(b)
    assert ia["n_leaves"] == ib["n_leaves"] and ia["bvh_depth"] == ib["bvh_depth"]
    uv = np.random.default_rng(11).uniform(0, 1, (20000, 2)).astype(np.float32)
    pa, ta = gpu.primary_hits(a, uv)
    pb, tb = gpu.primary_hits(b, uv)
    assert np.array_equal(ta.view(np.uint32), tb.view(np.uint32))
    assert (pa == pb).mean() >= 0.999
    pa, ta = gpu.trace_rays(a, fx["rays"])
    pb, tb = gpu.trace_rays(b, fx["rays"])
    assert np.array_equal(ta.view(np.uint32), tb.view(np.uint32))
    assert (pa == pb).mean() >= 0.999
    gpu.free(a)
    gpu.free(b)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name,engine", [("cornell_box", A.ENGINE_WAVEFRONT),
                                         ("cloud2k", A.ENGINE_WAVEFRONT),
                                         ("prims_mix", A.ENGINE_MEGAKERNEL),
                                         ("cloud2k", A.ENGINE_MEGAKERNEL)])
def test_device_traversal_tree_renders_the_same_image(gpu, name, engine, mode):
    scene, fx = load_golden(name)
    wd, ht, _, depth = (int(x) for x in fx["settings"])
    st = RenderSettings(width=wd, height=ht, samples=4, max_depth=depth, pathtrace=True,
                        pathtrace_bounces=depth, engine=engine)
    a, b = upload_both(gpu, scene, fx["nodes"], mode)
    assert same_pixels(gpu.render(a, st), gpu.render(b, st)) >= 0.999
    gpu.free(a)
    gpu.free(b)


@pytest.mark.parametrize("mode", MODES)
def test_device_traversal_tree_on_the_full_mesh(gpu, mode):
    """The 1,310,720-triangle mesh box, the workload the modes are for: the
    same hit distances for 50,000 camera rays, a window of the frame equal
    pixel for pixel but for rounding ties, fewer node visits per ray."""
    from pencil_b200.renderer import RenderStats
    w = W.mesh_box()
    nodes, _ = w.scene.build_bvh()
    a, b = upload_both(gpu, w.scene, nodes, mode)
    uv = np.random.default_rng(9).uniform(0, 1, (50000, 2)).astype(np.float32)
    pa, ta = gpu.primary_hits(a, uv)
    pb, tb = gpu.primary_hits(b, uv)
    assert np.array_equal(ta.view(np.uint32), tb.view(np.uint32))
    assert (pa == pb).mean() >= 0.999
    st = w.settings
    st.samples = 2
    win = (384, 384, 256, 256)
    imgs, visits = [], []
    for sid in (a, b):
        cnt = RenderStats()
        st.count_rays, st.count_nodes = True, True
        imgs.append(gpu.render_window(sid, st, win, stats=cnt))
        st.count_rays, st.count_nodes = False, False
        visits.append(cnt.ext_node_visits / max(1, cnt.extension_rays))
    print(f"mesh window, mode {mode}: {same_pixels(*imgs):.6f} of pixels equal; wide-node "
          f"visits per extension ray {visits[0]:.1f} (uploaded tree) vs {visits[1]:.1f}")
    assert same_pixels(*imgs) >= 0.999
    assert visits[1] < visits[0]
    gpu.free(a)
    gpu.free(b)


def test_traversal_tree_rejects_unknown_modes(gpu):
    assert gpu.lib.pgpu_set_traversal_tree(gpu.h, 3) == A.ERR_INVALID_ARG
    assert gpu.lib.pgpu_set_traversal_tree(gpu.h, -1) == A.ERR_INVALID_ARG
