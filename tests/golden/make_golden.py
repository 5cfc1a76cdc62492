"""Generate the golden fixtures of tests/golden from the reference renderer.

Run in a checkout next to the reference project (its sources and its own
golden PNGs); needs oracle/_ref/pencil_ref, built by
`make -C oracle REF_SRC=/path/to/pencil/src`:

    python tests/golden/make_golden.py --ref /path/to/pencil

Writes, for each fixture scene:
  scenes/<name>.bin   the scene (PGPUSCN1 format): the reference's parser output
                      for its example scenes, seeded synthetic scenes otherwise
  ref_<name>.npz      from the reference binary: stored primitive state, the
                      BVH in DFS pre-order and its depth, small path-traced and
                      Whitted HDR renders with their trace-call counts, closest
                      hits of seeded random rays, and camera rays of seeded
                      image-plane points
and png_goldens.json: digests of the reference's own golden PNGs
(tests/three_spheres.png, tests/shapes.png: SHA-256 of the decoded RGB;
tests/cornell_box.png: a seeded sample of pixels, since the current code
reproduces it to within 1 LSB only), and config_pins.json: SHA-256 digests
of the reference renderer's HDR output (and BVH) on the benchmark
configurations' own scenes at their configured image sizes (`--only configs`
writes just this file).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from pencil_b200 import _abi as A  # noqa: E402
from pencil_b200 import workloads as W  # noqa: E402
from pencil_b200.scene import CameraArgs, Light, Material, Scene  # noqa: E402

PECL_SCENES = ["three_spheres", "shapes", "cornell_box"]


def prims_mix() -> Scene:
    """Every primitive kind, every material kind, every light kind Pencil has."""
    s = Scene()
    s.background = (0.1, 0.12, 0.2)
    s.ambient = (0.04, 0.04, 0.05)
    gray = s.add_material(Material.diffuse((0.6, 0.6, 0.6), spec=0.2, shininess=16.0))
    red = s.add_material(Material.diffuse((0.8, 0.2, 0.1), spec=0.5, shininess=64.0))
    metal = s.add_material(Material.metal((0.9, 0.85, 0.8), 0.05))
    rough = s.add_material(Material.metal((0.7, 0.7, 0.9), 1.0))
    glass = s.add_material(Material.dielectric(1.5, (0.95, 0.97, 1.0)))
    blue = s.add_material(Material.diffuse((0.1, 0.3, 0.8)))
    lamp = s.add_material(Material(A.MAT_DIFFUSE, (0.0, 0.0, 0.0), (4.0, 3.5, 3.0)))
    s.add_plane((0, -1, 0), (0, 1, 0), gray)
    s.add_sphere((-1.5, 0, 0.5), 1.0, red)
    s.add_sphere((1.3, -0.3, -0.4), 0.7, glass)
    s.add_sphere((0.2, 1.4, 1.2), 0.5, metal)
    s.add_sphere((2.4, 1.5, 2.0), 0.3, lamp)
    s.add_cube((0.0, -0.55, -1.2), 0.45, rough)
    s.add_cylinder((-2.6, -0.2, -1.0), (0.2, 1.0, 0.1), 0.35, 1.6, blue)
    s.add_cone((2.6, 0.8, -0.8), (0.0, 1.0, 0.0), 0.5, 1.4, red)
    s.add_cone((-0.5, 1.2, -1.8), (0.3, -1.0, 0.2), 0.4, 1.0, metal)
    s.add_quad((-3, -1, 3), (3, -1, 3), (3, 3, 3), (-3, 3, 3), gray)
    s.add_triangle((-0.8, 1.6, -0.5), (0.6, 1.9, -0.2), (-0.1, 2.6, 0.4), glass)
    s.add_light(Light.point((4, 6, -4), (0.9, 0.9, 0.85), 0.5))
    s.add_light(Light.point((-4, 3, -3), (0.3, 0.3, 0.45), 0.0))
    s.add_light(Light.directional((0.3, -1.0, 0.4), (0.2, 0.2, 0.2)))
    s.add_light(Light.point((2.4, 1.5, 2.0), (4.0, 3.5, 3.0), 0.15, True))
    s.camera = CameraArgs((0.5, 1.8, -7.0), (0.0, 0.3, 0.0), (0, 1, 0), 55.0, 4.0 / 3.0)
    return s


def no_quad_lights(s: Scene) -> Scene:
    """The reference has no area lights: its emissive quads are reached by
    BSDF sampling only. Drop quad lights for the reference side."""
    s.lights = [l for l in s.lights if l.kind != A.LIGHT_QUAD]
    return s


def synthetic() -> dict[str, tuple[Scene, tuple[int, int, int, int]]]:
    """name -> (scene, (width, height, samples n, depth))"""
    out = {}
    out["c1"] = (W.three_spheres_pt(80, 60, 2, 8).scene, (80, 60, 2, 8))
    out["cloud2k"] = (W.sphere_cloud(2000, 96, 54, 2, 8, seed=7).scene, (96, 54, 2, 8))
    out["prims_mix"] = (prims_mix(), (64, 48, 2, 6))
    out["mesh_small"] = (no_quad_lights(W.mesh_box(subdiv=2, width=48, height=48).scene),
                         (48, 48, 2, 6))
    out["adjoint_small"] = (no_quad_lights(W.adjoint_box(60, 48, 48, 2, 4, seed=9)[0].scene),
                            (48, 48, 2, 4))
    return out


def fixture(name: str, scene: Scene, wh: tuple[int, int, int, int], rng) -> dict:
    W_, H_, n, depth = wh
    prims, nodes, tdepth = O.ref_dump(scene)
    d = {"prims": prims, "nodes": nodes, "depth": np.int32(tdepth),
         "settings": np.array([W_, H_, n, depth], np.int32)}
    for tag, pt in (("pt", True), ("wh", False)):
        img, info = O.ref_render(scene, W_, H_, n, depth, pt, threads=8)
        d[f"hdr_{tag}"] = img
        d[f"rays_{tag}"] = np.int64(info["rays"])
    # closest hits of seeded rays: camera-like rays and rays from inside the scene
    lo = np.minimum(nodes[0]["bmin"], 50.0) if len(nodes) else np.zeros(3)
    hi = np.maximum(nodes[0]["bmax"], -50.0) if len(nodes) else np.ones(3)
    lo = np.clip(lo, -50, 50)
    hi = np.clip(hi, -50, 50)
    k = 2048
    org = rng.uniform(lo, hi, size=(k, 3))
    dirs = rng.normal(size=(k, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = np.concatenate([org, dirs], 1).astype(np.float32)
    uv = rng.uniform(0, 1, size=(k, 2)).astype(np.float32)
    cam = O.ref_camrays(scene, uv)
    rays = np.concatenate([rays, cam]).astype(np.float32)
    prim, t = O.ref_hits(scene, rays)
    d.update({"rays": rays, "hit_prim": prim, "hit_t": t, "uv": uv, "cam_rays": cam})
    return d


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def config_pins() -> dict:
    """Reference renders of the benchmark configurations' scenes.

    c1_pt / c1_wh  three spheres, 320x240, n=2, depth 8 (path tracer / Whitted)
    c2_n1          the 100k-sphere cloud at its full 1280x720 frame, depth 8,
                   n=1 (the configured n=4 costs the reference 16x longer; the
                   sample loop, jitter and seeding are the same code at any n)
    c3_128         the full 1,310,720-triangle mesh box (the reference reaches
                   its emitter by BSDF sampling only), 128x128, n=1, depth 12
    c5_pt          the adjoint box (1,000 spheres), 512x512, n=4, depth 6
    Each entry: the settings, the SHA-256 of the HDR floats, their mean, the
    trace-call count and the SHA-256 of the reference's BVH node table."""
    cases = {
        "c1_pt": (W.three_spheres_pt(320, 240, 2, 8).scene, (320, 240, 2, 8), True),
        "c1_wh": (W.three_spheres_pt(320, 240, 2, 8).scene, (320, 240, 2, 8), False),
        "c2_n1": (W.sphere_cloud().scene, (1280, 720, 1, 8), True),
        "c3_128": (no_quad_lights(W.mesh_box().scene), (128, 128, 1, 12), True),
        "c5_pt": (no_quad_lights(W.adjoint_box()[0].scene), (512, 512, 4, 6), True),
    }
    out = {}
    for name, (scene, (w, h, n, depth), pt) in cases.items():
        _, nodes, tdepth = O.ref_dump(scene)
        img, info = O.ref_render(scene, w, h, n, depth, pt, threads=8)
        out[name] = {"settings": [w, h, n, depth], "pathtrace": pt, "hdr_sha256": _sha(img),
                     "hdr_mean": float(img.astype(np.float64).mean()),
                     "rays": int(info["rays"]), "nodes_sha256": _sha(nodes),
                     "bvh_depth": int(tdepth)}
        print("pinned", name, out[name]["hdr_mean"])
    return out


def png_goldens(ref_root: Path) -> dict:
    from PIL import Image
    rng = np.random.default_rng(11)
    out = {}
    for name in PECL_SCENES:
        png = ref_root / "tests" / f"{name}.png"
        px = np.asarray(Image.open(png).convert("RGB"))
        entry = {"shape": list(px.shape),
                 "sha256": hashlib.sha256(np.ascontiguousarray(px).tobytes()).hexdigest()}
        if name == "cornell_box":
            idx = rng.choice(px.shape[0] * px.shape[1], size=5000, replace=False)
            entry["sample_index"] = idx.astype(int).tolist()
            entry["sample_rgb"] = px.reshape(-1, 3)[idx].astype(int).tolist()
        out[name] = entry
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True,
                    help="root of the reference project (holds src/, examples/, tests/)")
    ap.add_argument("--only", choices=["configs"], default=None,
                    help="write only config_pins.json")
    a = ap.parse_args()
    ref_root = Path(a.ref)
    if not O.ref_available():
        raise SystemExit("oracle/_ref/pencil_ref is missing: run `make -C oracle` first")
    if a.only == "configs":
        (HERE / "config_pins.json").write_text(json.dumps(config_pins(), indent=1))
        print("wrote config_pins.json")
        return
    (HERE / "scenes").mkdir(exist_ok=True)
    rng = np.random.default_rng(1234)
    scenes = {}
    meta = {}
    for name in PECL_SCENES:
        path = HERE / "scenes" / f"{name}.bin"
        info = O.ref_parse(ref_root / "examples" / f"{name}.pecl", path)
        meta[name] = info
        scenes[name] = (Scene.read(path), (64, 48, 2, min(info["depth"], 8)))
    for name, (s, wh) in synthetic().items():
        s.write(HERE / "scenes" / f"{name}.bin")
        scenes[name] = (Scene.read(HERE / "scenes" / f"{name}.bin"), wh)
    for name, (s, wh) in scenes.items():
        np.savez_compressed(HERE / f"ref_{name}.npz", **fixture(name, s, wh, rng))
        print("wrote", name)
    gold = png_goldens(ref_root)
    for name in PECL_SCENES:
        gold[name]["render"] = meta[name]
    (HERE / "png_goldens.json").write_text(json.dumps(gold))
    print("wrote png_goldens.json")
    (HERE / "config_pins.json").write_text(json.dumps(config_pins(), indent=1))
    print("wrote config_pins.json")


if __name__ == "__main__":
    main()
