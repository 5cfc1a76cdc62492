"""Pencil's own render path with the --gpu bridge, end to end: Pencil's .pecl
parser and BVH (compiled from the reference sources into
oracle/_ref/pencil_gpu_demo) hand the scene to libpencil_gpu.so through
pencil_b200/bridge/pencil_gpu_bridge.hpp. Compared with Pencil's CPU render
of the same file (oracle/_ref/pencil_ref). Skipped where those binaries were
not built (they need the reference sources at build time)."""
from __future__ import annotations

import json
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from pencil_b200.scene import Scene

pytestmark = pytest.mark.gpu

DEMO = O.HERE / "_ref" / "pencil_gpu_demo"

# A scene written for this test in Pencil's scene language.
PECL = """
bg: <10, 12, 20>
amb: <4, 4, 5>
cmra {
  pos: <1, 2.2, -7>
  aim: <0, 0.6, 0>
  up: <0, 1, 0>
  fov: 50
}
mat { clr: <60, 60, 62>, spc: 10, shn: 8 }
plane { pos: <0, 0, 0>, nrm: <0, 1, 0> }
mat { clr: <85, 25, 20>, spc: 40, shn: 32 }
sphere { pos: <-1.6, 0.8, 0.3>, rad: 0.8 }
mat { clr: <96, 96, 98>, ior: 1.45 }
sphere { pos: <0.7, 0.6, -0.6>, rad: 0.6 }
mat { clr: <80, 80, 85>, rfl: 100, fuz: 4 }
cube { pos: <1.9, 0.5, 0.9>, size: 0.5 }
mat { clr: <20, 55, 85> }
cylinder { pos: <-0.2, 0.5, 1.6>, ax: <0, 1, 0>, rad: 0.35, h: 1.0 }
mat { clr: <75, 70, 20> }
cone { apex: <2.6, 1.4, -0.5>, ax: <0, 1, 0>, rad: 0.4, h: 1.2 }
light { type: point, pos: <3, 5, -3>, clr: <95, 95, 90> }
light { type: point, pos: <-3, 3, -2>, clr: <30, 30, 40>, radius: 0 }
render { size: 96 72, spp: 2, depth: 6 }
"""


@pytest.fixture(scope="module")
def pecl(tmp_path_factory):
    if not (DEMO.exists() and O.ref_available()):
        pytest.skip("oracle/_ref binaries not built")
    p = tmp_path_factory.mktemp("pecl") / "bridge_scene.pecl"
    p.write_text(PECL)
    return p


def run_demo(pecl: Path, out: Path, exact: bool, pathtrace: bool) -> dict:
    env = dict(os.environ, PENCIL_GPU_EXACT="1" if exact else "0")
    args = [str(DEMO), str(pecl), str(out)] + (["--pathtrace"] if pathtrace else [])
    proc = subprocess.run(args, capture_output=True, text=True, env=env, timeout=120)
    assert proc.returncode == 0, proc.stderr
    return json.loads(proc.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("pathtrace", [True, False])
def test_bridge_reproduces_pencil_render(pecl, tmp_path, pathtrace):
    info = O.ref_parse(pecl, tmp_path / "scene.bin")
    w, h, n, d = info["width"], info["height"], info["samples"], info["depth"]
    gpu = run_demo(pecl, tmp_path / "gpu.f32", True, pathtrace)
    img = np.fromfile(tmp_path / "gpu.f32", np.float32).reshape(h, w, 3)
    scene = Scene.read(tmp_path / "scene.bin")
    ref, rinfo = O.ref_render(scene, w, h, n, d, pathtrace)
    rel = np.abs(img.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-3)
    assert (rel > 1e-4).mean() <= 0.005
    assert gpu["rays"] == rinfo["rays"]      # Pencil's ray count, reproduced


def test_bridge_production_engine(pecl, tmp_path):
    info = O.ref_parse(pecl, tmp_path / "scene.bin")
    w, h = info["width"], info["height"]
    run_demo(pecl, tmp_path / "gpu.f32", False, True)
    img = np.fromfile(tmp_path / "gpu.f32", np.float32).reshape(h, w, 3)
    scene = Scene.read(tmp_path / "scene.bin")
    from pencil_b200.renderer import RenderSettings
    st = RenderSettings(width=w, height=h, samples=info["samples"], pathtrace=True,
                        pathtrace_bounces=info["depth"])
    ref, _, _ = O.Oracle(scene).render_split(st)
    rel = np.abs(img.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-3)
    assert (rel > 1e-4).mean() <= 0.005
