"""The oracle and the host-side BVH builder pinned against the reference.

Fixtures in tests/golden were produced by the reference renderer compiled
from its own sources (tests/golden/make_golden.py); the PNG digests are those
of the reference project's own golden images. Integer/byte/index results and
HDR floats must match bit for bit.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import GOLDEN_SCENES, load_golden, png_goldens
from oracle import oracle as O
from pencil_b200.renderer import RenderSettings


def settings_of(fx, pathtrace: bool) -> RenderSettings:
    w, h, n, depth = (int(x) for x in fx["settings"])
    return RenderSettings(width=w, height=h, samples=n, max_depth=depth, pathtrace=pathtrace,
                          pathtrace_bounces=depth)


@pytest.mark.parametrize("name", GOLDEN_SCENES)
def test_stored_primitive_state(name):
    scene, fx = load_golden(name)
    assert scene.unified_prims().tobytes() == fx["prims"].tobytes()


@pytest.mark.parametrize("name", GOLDEN_SCENES)
def test_bvh_builder_matches_reference_tree(name):
    scene, fx = load_golden(name)
    nodes, depth = scene.build_bvh()
    assert depth == int(fx["depth"])
    assert nodes.tobytes() == fx["nodes"].tobytes()


@pytest.mark.parametrize("name", GOLDEN_SCENES)
@pytest.mark.parametrize("mode", ["pt", "wh"])
def test_oracle_render_bit_exact(name, mode):
    scene, fx = load_golden(name)
    orc = O.Oracle(scene, fx["nodes"], fx["prims"])
    img, _, cnt = orc.render(settings_of(fx, mode == "pt"))
    ref = fx[f"hdr_{mode}"]
    assert img.shape == ref.shape
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    assert int(cnt[O.CNT_REFERENCE_RAYS]) == int(fx[f"rays_{mode}"])


@pytest.mark.parametrize("name", GOLDEN_SCENES)
def test_oracle_closest_hits_bit_exact(name):
    scene, fx = load_golden(name)
    orc = O.Oracle(scene, fx["nodes"], fx["prims"])
    prim, t = orc.trace_rays(fx["rays"])
    assert np.array_equal(prim, fx["hit_prim"])
    assert np.array_equal(t.view(np.uint32), fx["hit_t"].view(np.uint32))
    assert (prim >= 0).sum() > 0


@pytest.mark.parametrize("name", GOLDEN_SCENES)
def test_oracle_camera_rays_bit_exact(name):
    scene, fx = load_golden(name)
    orc = O.Oracle(scene, fx["nodes"], fx["prims"])
    rays = orc.camera_rays(fx["uv"])
    assert np.array_equal(rays.view(np.uint32), fx["cam_rays"].view(np.uint32))


@pytest.mark.parametrize("name", ["three_spheres", "shapes", "cornell_box"])
def test_reference_png_goldens(name):
    """Pencil's own golden PNGs (Whitted mode, ACES + gamma 2.2, 8 bit):
    three_spheres and shapes byte-exact, cornell_box within 1 LSB."""
    scene, fx = load_golden(name)
    g = png_goldens()[name]
    r = g["render"]
    st = RenderSettings(width=r["width"], height=r["height"], samples=r["samples"],
                        max_depth=r["depth"], pathtrace=False)
    img, _, _ = O.Oracle(scene, fx["nodes"], fx["prims"]).render(st)
    px = O.rgb8(img, tonemap=1)
    assert list(px.shape) == g["shape"]
    if "sample_index" in g:
        got = px.reshape(-1, 3)[np.asarray(g["sample_index"])].astype(int)
        diff = np.abs(got - np.asarray(g["sample_rgb"]))
        assert diff.max() <= 1
    else:
        assert hashlib.sha256(np.ascontiguousarray(px).tobytes()).hexdigest() == g["sha256"]


def test_counter_rng_seed_is_deterministic_and_nonzero():
    seeds = {O.path_seed(i, j, s) for i in range(8) for j in range(8) for s in range(16)}
    assert 0 not in seeds
    assert len(seeds) == 8 * 8 * 16
    assert O.path_seed(3, 4, 5, 7) == O.path_seed(3, 4, 5, 7)
    assert O.path_seed(3, 4, 5, 7) != O.path_seed(3, 4, 5, 8)
