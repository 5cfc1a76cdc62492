"""pgpu_build_bvh_device: a linear BVH built on the GPU in Pencil's node-table
format. It is a different tree from Pencil's SAH tree, so the checks are on
its structure and on what it finds: a valid DFS pre-order table with every
primitive in one leaf (the upload validates it too), the same closest-hit
distances as Pencil's tree for camera and random rays (the primitive may
differ only between surfaces at exactly the same distance), and renders
that agree with those on Pencil's tree."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN_SCENES, load_golden
from pencil_b200 import _abi as A
from pencil_b200 import workloads as W
from pencil_b200.renderer import RenderSettings

pytestmark = pytest.mark.gpu


def check_table(nodes: np.ndarray, n_prims: int) -> int:
    """Validates DFS pre-order links and leaves; returns the depth."""
    assert len(nodes) == max(2 * n_prims - 1, 0)
    if n_prims == 0:
        return 0
    size = np.zeros(len(nodes), np.int64)
    for k in range(len(nodes) - 1, -1, -1):
        nd = nodes[k]
        if nd["left"] < 0:
            size[k] = 1
            continue
        assert nd["left"] == k + 1 and nd["right"] == nd["left"] + size[nd["left"]]
        size[k] = 1 + size[nd["left"]] + size[nd["right"]]
        for c in (nd["left"], nd["right"]):        # parent box holds the child's
            assert np.all(nodes[c]["bmin"] >= nd["bmin"]) and np.all(nodes[c]["bmax"] <= nd["bmax"])
    assert size[0] == len(nodes)
    leaves = nodes[nodes["left"] < 0]["right"]
    assert sorted(leaves.tolist()) == list(range(n_prims))
    level = np.zeros(len(nodes), np.int64)
    level[0] = 1
    for k in range(len(nodes)):
        if nodes[k]["left"] >= 0:
            level[nodes[k]["left"]] = level[nodes[k]["right"]] = level[k] + 1
    return int(level.max())


@pytest.mark.parametrize("name", GOLDEN_SCENES)
def test_device_tree_is_valid_and_finds_the_same_hits(gpu, name):
    scene, fx = load_golden(name)
    nodes, depth = gpu.build_bvh_device(scene)
    assert check_table(nodes, scene.n_unified) == depth
    sid_host = gpu.upload(scene, fx["nodes"])
    sid_dev = gpu.upload(scene, nodes)
    rng = np.random.default_rng(5)
    uv = rng.uniform(0, 1, (20000, 2)).astype(np.float32)
    ph, th = gpu.primary_hits(sid_host, uv)
    pd, td = gpu.primary_hits(sid_dev, uv)
    assert np.array_equal(th.view(np.uint32), td.view(np.uint32))
    assert (ph == pd).mean() >= 0.999          # ties at equal distance may pick another
    ph, th = gpu.trace_rays(sid_host, fx["rays"])
    pd, td = gpu.trace_rays(sid_dev, fx["rays"])
    assert np.array_equal(th.view(np.uint32), td.view(np.uint32))
    assert (ph == pd).mean() >= 0.999
    gpu.free(sid_host)
    gpu.free(sid_dev)


def test_device_tree_edge_cases(gpu):
    from pencil_b200.scene import Material, Scene
    s = Scene()
    assert len(gpu.build_bvh_device(s)[0]) == 0
    m = s.add_material(Material.diffuse((0.5, 0.5, 0.5)))
    s.add_sphere((0, 0, 0), 1.0, m)
    nodes, depth = gpu.build_bvh_device(s)
    assert len(nodes) == 1 and depth == 1
    for _ in range(40):                         # identical centres: keys tie on Morton code
        s.add_sphere((1.0, 2.0, 3.0), 0.5, m)
    nodes, depth = gpu.build_bvh_device(s)
    assert check_table(nodes, s.n_unified) == depth


def test_device_tree_renders_the_sphere_cloud_and_the_mesh(gpu):
    for wl, size in ((W.sphere_cloud(), (320, 180)), (W.mesh_box(subdiv=5), (128, 128))):
        st = wl.settings
        st.width, st.height = size
        st.samples = 2
        nodes, depth = gpu.build_bvh_device(wl.scene)
        assert check_table(nodes, wl.scene.n_unified) == depth
        a = gpu.upload(wl.scene)
        b = gpu.upload(wl.scene, nodes)
        ia, ib = gpu.render(a, st), gpu.render(b, st)
        same = np.all(ia.view(np.uint32) == ib.view(np.uint32), axis=2).mean()
        assert same >= 0.999, same
        gpu.free(a)
        gpu.free(b)


# ---- Pencil's SAH tree built on the device (pgpu_build_bvh_device_sah) ----------------
@pytest.mark.parametrize("name", GOLDEN_SCENES)
def test_device_sah_tree_valid_and_hits_equal(gpu, name):
    """Valid table; the same hits as the reference's tree; node for node the
    reference's tree except where a median split meets tied centroid keys."""
    scene, fx = load_golden(name)
    nodes, depth = gpu.build_bvh_device(scene, method="sah")
    assert check_table(nodes, scene.n_unified) == depth
    same = np.mean([a.tobytes() == b.tobytes() for a, b in zip(nodes, fx["nodes"])])
    print(f"{name}: {same:.4f} of nodes equal to the reference tree's")
    sid_host = gpu.upload(scene, fx["nodes"])
    sid_dev = gpu.upload(scene, nodes)
    ph, th = gpu.trace_rays(sid_host, fx["rays"])
    pd, td = gpu.trace_rays(sid_dev, fx["rays"])
    assert np.array_equal(th.view(np.uint32), td.view(np.uint32))
    assert (ph == pd).mean() >= 0.999
    gpu.free(sid_host)
    gpu.free(sid_dev)


@pytest.mark.parametrize("wl_name", ["sphere_cloud", "cloud_seed3", "sphere_batch"])
def test_device_sah_equals_reference_tree_without_ties(gpu, wl_name):
    """Random sphere scenes have no tied centroid keys: the device build is
    Pencil's SAH tree node for node (the host build equals the reference's,
    test_oracle_golden.py / test_oracle_config_pins.py)."""
    import time
    if wl_name == "sphere_cloud":
        scene = W.sphere_cloud().scene
    elif wl_name == "cloud_seed3":
        scene = W.sphere_cloud(20000, 64, 64, 1, 8, seed=3).scene
    else:
        scene = W.sphere_batch(n_scenes=3, seed=8)[2].scene
    t0 = time.perf_counter()
    host, hdepth = scene.build_bvh()
    t1 = time.perf_counter()
    gpu.build_bvh_device(scene, method="sah")
    t2 = time.perf_counter()
    dev, ddepth = gpu.build_bvh_device(scene, method="sah")
    t3 = time.perf_counter()
    print(f"{wl_name}: {scene.n_unified} primitives, host SAH {1e3 * (t1 - t0):.1f} ms, "
          f"device SAH {1e3 * (t3 - t2):.1f} ms")
    assert ddepth == hdepth
    assert dev.tobytes() == host.tobytes()


def test_device_sah_on_the_full_mesh(gpu):
    """The 1,310,720-triangle mesh box: symmetric triangles tie in median
    splits, so the trees differ in places; the table is valid, its depth is
    the host tree's give or take, and it finds the same hit distances (and,
    but for surfaces at exactly equal distances, the same primitives)."""
    import time
    w = W.mesh_box()
    host, hdepth = w.scene.build_bvh()
    gpu.build_bvh_device(w.scene, method="sah")
    t0 = time.perf_counter()
    dev, ddepth = gpu.build_bvh_device(w.scene, method="sah")
    ms = 1e3 * (time.perf_counter() - t0)
    same = np.mean(dev["left"] == host["left"])
    print(f"mesh: device SAH {ms:.1f} ms, depth {ddepth} (host {hdepth}), "
          f"{same:.4f} of nodes with the host tree's shape")
    assert check_table(dev, w.scene.n_unified) == ddepth
    assert abs(ddepth - hdepth) <= 4
    sa, sb = gpu.upload(w.scene, host), gpu.upload(w.scene, dev)
    uv = np.random.default_rng(9).uniform(0, 1, (50000, 2)).astype(np.float32)
    pa, ta = gpu.primary_hits(sa, uv)
    pb, tb = gpu.primary_hits(sb, uv)
    assert np.array_equal(ta.view(np.uint32), tb.view(np.uint32))
    assert (pa == pb).mean() >= 0.999
    gpu.free(sa)
    gpu.free(sb)


def test_device_sah_edge_cases(gpu):
    from pencil_b200.scene import Material, Scene
    s = Scene()
    assert len(gpu.build_bvh_device(s, method="sah")[0]) == 0
    m = s.add_material(Material.diffuse((0.5, 0.5, 0.5)))
    s.add_sphere((0, 0, 0), 1.0, m)
    assert len(gpu.build_bvh_device(s, method="sah")[0]) == 1
    for k in range(3):                          # 2 to 4 primitives: the root is small
        s.add_sphere((k + 1.0, 0.5 * k, 0), 0.5, m)
        nodes, depth = gpu.build_bvh_device(s, method="sah")
        host, hdepth = s.build_bvh()
        assert nodes.tobytes() == host.tobytes() and depth == hdepth
    for _ in range(40):                         # identical boxes: every split is a median split
        s.add_sphere((1.0, 2.0, 3.0), 0.5, m)
    nodes, depth = gpu.build_bvh_device(s, method="sah")
    assert check_table(nodes, s.n_unified) == depth
    s.add_plane((0, -1, 0), (0, 1, 0), m)       # a +-1e6 box: the root's bins all fall together
    nodes, depth = gpu.build_bvh_device(s, method="sah")
    assert check_table(nodes, s.n_unified) == depth
