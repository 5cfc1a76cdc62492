"""Shared fixtures. Tests marked `gpu` need a CUDA device and run through the
C-ABI of libpencil_gpu.so; everything else runs on the CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))

GOLDEN_SCENES = ["three_spheres", "shapes", "cornell_box", "c1", "cloud2k", "prims_mix",
                 "mesh_small", "adjoint_small"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")


def load_golden(name: str):
    """(scene, fixture dict) of a golden scene."""
    from pencil_b200.scene import Scene
    scene = Scene.read(GOLDEN / "scenes" / f"{name}.bin")
    with np.load(GOLDEN / f"ref_{name}.npz") as z:
        fx = {k: z[k] for k in z.files}
    return scene, fx


def png_goldens() -> dict:
    return json.loads((GOLDEN / "png_goldens.json").read_text())


@pytest.fixture(scope="session")
def gpu():
    from pencil_b200.renderer import GpuContext
    ctx = GpuContext(0)
    yield ctx
    ctx.close()
