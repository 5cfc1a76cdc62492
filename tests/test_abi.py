"""The C-ABI library: it loads, exports every function include/pencil_gpu.h
declares, and its host-only entry points behave (no GPU needed)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from pencil_b200 import _abi as A
from pencil_b200.scene import Scene, make_prim, normalized

HEADER = Path(__file__).resolve().parent.parent / "include" / "pencil_gpu.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pgpu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = A.load()
    names = declared_functions()
    assert len(names) >= 16
    for n in names:
        assert hasattr(lib, n), f"{n} declared in pencil_gpu.h but not exported"
    assert set(names) == set(A.EXPORTS), "ctypes binding out of step with the header"


def test_abi_version_and_record_sizes():
    lib = A.load()
    assert lib.pgpu_abi_version() == A.ABI_VERSION == 2
    assert C.sizeof(A.Camera) == 52
    assert C.sizeof(A.RenderParams) == 68
    assert C.sizeof(A.Stats) == 152
    assert C.sizeof(A.SceneInfo) == 32


def test_null_context_is_rejected():
    lib = A.load()
    sid = C.c_int32(0)
    d = A.SceneDesc()
    assert lib.pgpu_upload_scene(None, C.byref(d), C.byref(sid)) == A.ERR_INVALID_ARG
    p = A.RenderParams()
    assert lib.pgpu_render(None, 1, C.byref(p), None, None, None) == A.ERR_INVALID_ARG
    assert lib.pgpu_free_scene(None, 1) == A.ERR_INVALID_ARG
    assert lib.pgpu_get_scene_info(None, 1, None) == A.ERR_INVALID_ARG
    assert lib.pgpu_last_error(None) == b"null context"
    assert lib.pgpu_set_stream(None, None) == A.ERR_INVALID_ARG


def test_create_reports_missing_device_with_a_status():
    """Without a CUDA device the library answers with an error code; it has
    no CPU fallback. With one, it creates a context."""
    lib = A.load()
    h = C.c_void_p()
    rc = lib.pgpu_create(0, C.byref(h))
    assert rc in (A.OK, A.ERR_CUDA)
    if rc == A.OK:
        lib.pgpu_destroy(h)
    assert lib.pgpu_create(-1, C.byref(h)) in (A.ERR_INVALID_ARG, A.ERR_CUDA)


def test_make_prim_repeats_constructor_arithmetic():
    p = make_prim(A.PRIM_PLANE, 2, (0, 1, 0), (1.0, 2.0, 2.0))
    assert p["material"][0] == 2
    assert np.array_equal(p["p"][0, 3:6], normalized((1.0, 2.0, 2.0)))
    c = make_prim(A.PRIM_CYLINDER, 0, (1, 2, 3), (0, 3, 4), c=None, s0=0.5, s1=3.0)
    assert np.array_equal(c["p"][0, 3:6], normalized((0, 3, 4)))
    assert c["p"][0, 6] == np.float32(0.5) and c["p"][0, 7] == np.float32(1.5)
    k = make_prim(A.PRIM_CONE, 0, (1, 2, 3), (0, 0, 2), s0=0.5, s1=2.0)
    assert np.array_equal(k["p"][0, 3:6], [0, 0, 1]) and k["p"][0, 7] == np.float32(2.0)
    lib = A.load()
    out = np.zeros(1, A.PRIM_DTYPE)
    assert lib.pgpu_make_prim(99, 0, None, None, None, 0.0, 0.0, A.ptr(out)) == A.ERR_INVALID_ARG
    assert lib.pgpu_make_prim(A.PRIM_SPHERE, 0, None, None, None, 1.0, 0.0,
                              A.ptr(out)) == A.ERR_INVALID_ARG


def test_build_bvh_edge_cases():
    s = Scene()
    nodes, depth = s.build_bvh()
    assert len(nodes) == 0 and depth == 0
    m = s.add_material(__import__("pencil_b200").Material.diffuse((0.5, 0.5, 0.5)))
    s.add_sphere((0, 0, 0), 1.0, m)
    nodes, depth = s.build_bvh()
    assert len(nodes) == 1 and depth == 1 and nodes[0]["left"] == -1 and nodes[0]["right"] == 0
    s.add_sphere((3, 0, 0), 1.0, m)
    nodes, depth = s.build_bvh()
    assert len(nodes) == 3 and depth == 2 and nodes[0]["left"] == 1
    # every primitive exactly once, DFS pre-order links
    for n in (5, 37, 1000):
        s2 = Scene()
        m2 = s2.add_material(__import__("pencil_b200").Material.diffuse((0.5, 0.5, 0.5)))
        rng = np.random.default_rng(n)
        s2.add_spheres(rng.uniform(-5, 5, (n, 3)), rng.uniform(0.1, 0.3, n),
                       np.full(n, m2, np.int32))
        nodes, depth = s2.build_bvh()
        assert len(nodes) == 2 * n - 1
        leaves = nodes[nodes["left"] < 0]["right"]
        assert sorted(leaves.tolist()) == list(range(n))
        inner = np.nonzero(nodes["left"] >= 0)[0]
        assert np.all(nodes["left"][inner] == inner + 1)
        assert np.all(nodes["right"][inner] > inner + 1)


def test_build_bvh_rejects_bad_mesh_indices():
    s = Scene()
    m = s.add_material(__import__("pencil_b200").Material.diffuse((0.5, 0.5, 0.5)))
    s.set_mesh(np.zeros((3, 3), np.float32), np.array([[0, 1, 5]], np.int32), m)
    with pytest.raises(A.GpuError):
        s.build_bvh()
