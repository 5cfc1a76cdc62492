"""The oracle pinned on the benchmark configurations' own scenes at their
configured image sizes.

tests/golden/config_pins.json holds SHA-256 digests of the reference
renderer's HDR output and BVH node table for the three-spheres scene at
320x240 (path tracer and Whitted), the 100k-sphere cloud at its full
1280x720 frame, the full 1,310,720-triangle mesh box and the 1,000-sphere
adjoint box at 512x512 (made by tests/golden/make_golden.py from the
reference compiled from its own sources). The oracle and the host SAH build
must reproduce every digest bit for bit; the GPU tests at these sizes
(test_gpu_configs.py) then compare the GPU core against the oracle.
"""
from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O
from pencil_b200 import workloads as W
from pencil_b200.renderer import RenderSettings

PINS = json.loads((GOLDEN / "config_pins.json").read_text())


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def scene_of(name: str):
    if name.startswith("c1"):
        return W.three_spheres_pt(320, 240, 2, 8).scene
    if name == "c2_n1":
        return W.sphere_cloud().scene
    if name == "c3_128":
        return W.mesh_box().scene         # the oracle's reference mode ignores quad lights
    if name == "c5_pt":
        return W.adjoint_box()[0].scene
    raise KeyError(name)


@pytest.mark.parametrize("name", sorted(PINS))
def test_oracle_reproduces_reference_at_config_size(name):
    pin = PINS[name]
    scene = scene_of(name)
    nodes, depth = scene.build_bvh()
    assert sha(nodes) == pin["nodes_sha256"], "host SAH build differs from the reference tree"
    assert depth == pin["bvh_depth"]
    w, h, n, d = pin["settings"]
    st = RenderSettings(width=w, height=h, samples=n, max_depth=d, pathtrace=pin["pathtrace"],
                        pathtrace_bounces=d)
    img, _, cnt = O.Oracle(scene, nodes).render(st)
    assert int(cnt[O.CNT_REFERENCE_RAYS]) == pin["rays"]
    assert sha(img) == pin["hdr_sha256"]
