"""Seeded random scenes checked live against the reference binary
(oracle/_ref/pencil_ref, built from the reference sources by
`make -C oracle`). Skipped where that binary is absent."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from pencil_b200 import _abi as A
from pencil_b200.renderer import RenderSettings
from pencil_b200.scene import CameraArgs, Light, Material, Scene

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference binary not built")


def random_scene(seed: int, n: int) -> Scene:
    rng = np.random.default_rng(seed)
    s = Scene()
    s.background = tuple(rng.uniform(0, 0.4, 3))
    s.ambient = tuple(rng.uniform(0, 0.1, 3))
    mats = []
    for _ in range(6):
        k = rng.integers(0, 3)
        alb = tuple(rng.uniform(0.1, 0.95, 3))
        if k == 0:
            mats.append(s.add_material(Material.diffuse(alb, spec=float(rng.uniform(0, 0.5)),
                                                        shininess=float(rng.uniform(4, 64)))))
        elif k == 1:
            mats.append(s.add_material(Material.metal(alb, float(rng.uniform(0, 1.0)))))
        else:
            mats.append(s.add_material(Material.dielectric(float(rng.uniform(1.1, 2.0)), alb)))
    emit = s.add_material(Material(A.MAT_DIFFUSE, (0.2, 0.2, 0.2), tuple(rng.uniform(1, 5, 3))))
    mats.append(emit)
    for _ in range(n):
        m = int(rng.choice(mats))
        c = rng.uniform(-4, 4, 3)
        kind = rng.integers(0, 7)
        if kind == 0:
            s.add_sphere(c, float(rng.uniform(0.1, 1.0)), m)
        elif kind == 1:
            s.add_triangle(c, c + rng.normal(size=3), c + rng.normal(size=3), m)
        elif kind == 2:
            s.add_cube(c, float(rng.uniform(0.1, 0.8)), m)
        elif kind == 3:
            s.add_cylinder(c, rng.normal(size=3), float(rng.uniform(0.1, 0.6)),
                           float(rng.uniform(0.2, 2.0)), m)
        elif kind == 4:
            s.add_cone(c, rng.normal(size=3), float(rng.uniform(0.1, 0.6)),
                       float(rng.uniform(0.2, 2.0)), m)
        elif kind == 5:
            d = rng.normal(size=3)
            s.add_quad(c, c + [d[0], 0, 0], c + [d[0], d[1], 0], c + [0, d[1], 0], m)
        else:
            # axis-aligned quad: flat boxes, shared-edge ties
            e = float(rng.uniform(0.5, 2))
            s.add_quad(c, c + [e, 0, 0], c + [e, 0, e], c + [0, 0, e], m)
    if seed % 2 == 0:
        s.add_plane((0, -5, 0), rng.normal(size=3) * 0.1 + [0, 1, 0], mats[0])
    s.add_light(Light.point(tuple(rng.uniform(-6, 6, 3)), tuple(rng.uniform(0.3, 1, 3)),
                            float(rng.choice([0.0, 0.5]))))
    s.add_light(Light.directional(tuple(rng.normal(size=3)), tuple(rng.uniform(0.1, 0.5, 3))))
    s.add_light(Light.point(tuple(rng.uniform(-3, 3, 3)), (1.0, 1.0, 1.0), 0.2, True))
    s.camera = CameraArgs(tuple(rng.uniform(-2, 2, 3) + [0, 2, -12]), (0, 0, 0), (0, 1, 0),
                          float(rng.uniform(35, 70)), 4.0 / 3.0)
    return s


@pytest.mark.parametrize("seed,n", [(1, 1), (2, 2), (3, 5), (4, 13), (5, 40), (6, 150),
                                    (7, 700)])
def test_bvh_and_state_match_reference(seed, n):
    s = random_scene(seed, n)
    prims, nodes, depth = O.ref_dump(s)
    mine, mdepth = s.build_bvh()
    assert s.unified_prims().tobytes() == prims.tobytes()
    assert mine.tobytes() == nodes.tobytes()
    assert mdepth == depth


def test_bvh_degenerate_inputs():
    """Coincident centroids, identical boxes and planes (the +-1e6 box)."""
    s = Scene()
    m = s.add_material(Material.diffuse((0.5, 0.5, 0.5)))
    for _ in range(20):
        s.add_sphere((1.0, 2.0, 3.0), 0.5, m)
    for k in range(9):
        s.add_plane((0, k, 0), (0, 1, 0), m)
    for k in range(7):
        s.add_sphere((k * 0.5, 0, 0), 0.1, m)
    prims, nodes, depth = O.ref_dump(s)
    mine, mdepth = s.build_bvh()
    assert mine.tobytes() == nodes.tobytes() and mdepth == depth


@pytest.mark.parametrize("seed", [11, 12, 13, 14])
@pytest.mark.parametrize("pathtrace", [True, False])
def test_oracle_render_matches_reference(seed, pathtrace):
    s = random_scene(seed, 60)
    st = RenderSettings(width=40, height=30, samples=2, max_depth=6, pathtrace=pathtrace,
                        pathtrace_bounces=6)
    img, _, cnt = O.Oracle(s).render(st)
    ref, info = O.ref_render(s, 40, 30, 2, 6, pathtrace)
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    assert int(cnt[O.CNT_REFERENCE_RAYS]) == info["rays"]


@pytest.mark.parametrize("seed", [15, 16, 17])
def test_oracle_mis_render_matches_reference(seed):
    """Path tracing with RenderSettings::mis (trace_path_mis): disc, point and
    directional lights, bit for bit, same ray count."""
    s = random_scene(seed, 60)
    st = RenderSettings(width=40, height=30, samples=2, max_depth=6, pathtrace=True,
                        pathtrace_bounces=6, mis=True)
    img, _, cnt = O.Oracle(s).render(st)
    ref, info = O.ref_render(s, 40, 30, 2, 6, True, mis=True)
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    assert int(cnt[O.CNT_REFERENCE_RAYS]) == info["rays"]
    plain, _, _ = O.Oracle(s).render(dataclasses.replace(st, mis=False))
    assert not np.array_equal(img, plain)        # the weights changed the image


@pytest.mark.parametrize("seed", [18, 19])
def test_oracle_tile_matches_reference_worker(seed):
    """The distributed worker's render_tile (src/distributed.hpp:380-434):
    Whitted trace, per-pixel seeds of the full image, half-pixel jitter."""
    s = random_scene(seed, 60)
    st = RenderSettings(width=48, height=36, samples=2, max_depth=5, pathtrace=False)
    for x, y, w, h in ((0, 0, 48, 36), (10, 7, 16, 12), (47, 35, 1, 1)):
        mine = O.Oracle(s).render_tile(st, x, y, w, h)
        ref = O.ref_tile(s, 48, 36, x, y, w, h, 2, 5)
        assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("seed", [21, 22])
def test_oracle_hits_match_reference(seed):
    s = random_scene(seed, 200)
    rng = np.random.default_rng(seed)
    org = rng.uniform(-6, 6, size=(3000, 3))
    d = rng.normal(size=(3000, 3))
    rays = np.concatenate([org, d / np.linalg.norm(d, axis=1, keepdims=True)], 1)
    rays = rays.astype(np.float32)
    prim, t = O.Oracle(s).trace_rays(rays)
    rp, rt = O.ref_hits(s, rays)
    assert np.array_equal(prim, rp)
    assert np.array_equal(t.view(np.uint32), rt.view(np.uint32))
