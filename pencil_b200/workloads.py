"""Seeded synthetic workloads of the benchmark configurations.

No public dataset is involved: every scene is generated from a numpy seed.

  three_spheres_pt   plane + red diffuse / mirror / glass spheres, one hard point
                     light; 320x240, n=2 (4 spp), depth 8
  sphere_cloud       100,000 random spheres (60/30/10 diffuse/metal/glass), one
                     directional light, sky 0.3; 1280x720, n=4 (16 spp), depth 8
  mesh_box           displaced icosphere (8 subdivisions, 1,310,720 triangles,
                     float32 vertices + int32 indices) in a box of 5 diffuse
                     walls with a 0.25x0.25 emissive quad in the ceiling, used
                     as an area light;
                     1024x1024, n=8 (64 spp), depth 12
  sphere_batch       256 sphere_cloud scenes of 10..50,000 spheres at
                     128/256/512 squared with 1/4/16/64 spp, depth 8
  adjoint_box        the mesh_box box with 1,000 small diffuse spheres, each its
                     own material; 512x512, n=4 (16 spp), depth 6
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _abi as A
from .renderer import RenderSettings
from .scene import CameraArgs, Light, Material, Scene


@dataclass
class Workload:
    name: str
    scene: Scene
    settings: RenderSettings


def three_spheres_pt(width: int = 320, height: int = 240, samples: int = 2,
                     depth: int = 8) -> Workload:
    s = Scene()
    s.background = (0.0, 0.0, 0.0)
    s.ambient = (0.05, 0.05, 0.05)
    floor = s.add_material(Material.diffuse((0.5, 0.5, 0.5)))
    red = s.add_material(Material.diffuse((0.8, 0.1, 0.1)))
    mirror = s.add_material(Material.metal((1.0, 1.0, 1.0), 0.0))
    glass = s.add_material(Material.dielectric(1.5, (1.0, 1.0, 1.0)))
    s.add_plane((0, 0, 0), (0, 1, 0), floor)
    s.add_sphere((-2.2, 1, 0), 1.0, red)
    s.add_sphere((0, 1, 0), 1.0, mirror)
    s.add_sphere((2.2, 1, 0), 1.0, glass)
    s.add_light(Light.point((5, 8, 5), (1.0, 1.0, 1.0), 0.0))
    s.camera = CameraArgs((0, 2, -8), (0, 1, 0), (0, 1, 0), 60.0, width / height)
    st = RenderSettings(width=width, height=height, samples=samples, max_depth=depth,
                        pathtrace=True, pathtrace_bounces=depth)
    return Workload("three_spheres_pt", s, st)


def _cloud(rng: np.random.Generator, n: int) -> Scene:
    s = Scene()
    s.background = (0.3, 0.3, 0.3)
    s.ambient = (0.0, 0.0, 0.0)
    centers = rng.uniform(-50.0, 50.0, size=(n, 3)).astype(np.float32)
    radii = np.exp(rng.uniform(np.log(0.05), np.log(0.5), size=n)).astype(np.float32)
    kind = rng.uniform(size=n)
    albedo = rng.uniform(0.1, 0.9, size=(n, 3)).astype(np.float32)
    fuzz = rng.uniform(0.0, 0.3, size=n).astype(np.float32)
    mats = np.zeros(n, A.MATERIAL_DTYPE)
    mats["kind"] = np.where(kind < 0.6, A.MAT_DIFFUSE, np.where(kind < 0.9, A.MAT_METAL,
                                                                A.MAT_DIELECTRIC))
    mats["albedo"] = np.where((mats["kind"] == A.MAT_DIELECTRIC)[:, None], 1.0, albedo)
    mats["reflectivity"] = np.where(mats["kind"] == A.MAT_METAL, np.float32(1.0) - fuzz, 0.0)
    mats["ior"] = np.where(mats["kind"] == A.MAT_DIELECTRIC, 1.5, 1.0)
    mats["shininess"] = 32.0
    mats["specular_color"] = 1.0
    s.add_material_array(mats)
    s.add_spheres(centers, radii, np.arange(n, dtype=np.int32))
    s.add_light(Light.directional((-1.0, -2.0, 1.0), (1.0, 1.0, 1.0)))
    return s


def sphere_cloud(n: int = 100_000, width: int = 1280, height: int = 720, samples: int = 4,
                 depth: int = 8, seed: int = 2) -> Workload:
    s = _cloud(np.random.default_rng(seed), n)
    s.camera = CameraArgs((0, 0, -120), (0, 0, 0), (0, 1, 0), 45.0, width / height)
    st = RenderSettings(width=width, height=height, samples=samples, max_depth=depth,
                        pathtrace=True, pathtrace_bounces=depth)
    return Workload("sphere_cloud", s, st)


def sphere_batch(n_scenes: int = 256, seed: int = 4, depth: int = 8) -> list[Workload]:
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        n = int(np.exp(rng.uniform(np.log(10), np.log(50_000))))
        res = int(rng.choice([128, 256, 512]))
        samples = int(rng.choice([1, 2, 4, 8]))
        s = _cloud(np.random.default_rng(1000 + k), n)
        s.camera = CameraArgs((0, 0, -120), (0, 0, 0), (0, 1, 0), 45.0, 1.0)
        st = RenderSettings(width=res, height=res, samples=samples, max_depth=depth,
                            pathtrace=True, pathtrace_bounces=depth, seed=k)
        out.append(Workload(f"sphere_batch_{k}", s, st))
    return out


# ---- mesh box -------------------------------------------------------------------
def icosphere(subdiv: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4**subdiv triangles, 10 * 4**subdiv + 2 vertices."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        nv = len(v)
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * nv + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // nv, uniq % nv
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1) + nv          # midpoint ids of edges ab, bc, ca
        ab, bc, ca = m[0], m[1], m[2]
        f = np.concatenate([np.stack([f[:, 0], ab, ca], 1), np.stack([ab, f[:, 1], bc], 1),
                            np.stack([ca, bc, f[:, 2]], 1), np.stack([ab, bc, ca], 1)])
        v = np.concatenate([v, mid])
    return v, f


def value_noise(p: np.ndarray, seed: int, octaves: int = 3, base_freq: float = 2.0,
                lattice: int = 64) -> np.ndarray:
    """Seeded 3-octave value noise in [-1, 1]: smooth-step trilinear
    interpolation of random lattice values, octave k at base_freq * 2**k with
    weight 0.5**k."""
    rng = np.random.default_rng(seed)
    total = np.zeros(len(p))
    norm = 0.0
    for k in range(octaves):
        grid = rng.uniform(-1.0, 1.0, size=(lattice, lattice, lattice))
        x = (p + 1.0) * base_freq * 2 ** k
        i0 = np.floor(x).astype(np.int64)
        fr = x - i0
        w = fr * fr * (3.0 - 2.0 * fr)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    g = grid[(i0[:, 0] + dx) % lattice, (i0[:, 1] + dy) % lattice,
                             (i0[:, 2] + dz) % lattice]
                    wx = w[:, 0] if dx else 1.0 - w[:, 0]
                    wy = w[:, 1] if dy else 1.0 - w[:, 1]
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    acc += g * wx * wy * wz
        total += acc * 0.5 ** k
        norm += 0.5 ** k
    return total / norm


def _box(s: Scene, emitter_radiance=(17.0, 12.0, 4.0)) -> None:
    """Unit box [0,1]^3 open at z=0: floor, ceiling, back (albedo 0.75), red
    left wall and green right wall (0.65 in their own channel, 0.05 in the
    others). The ceiling is four quads around a 0.25 x 0.25 opening at its
    centre, which the emissive quad fills (coplanar, facing down); that quad
    is also registered as a quad light. Keeping the emitter in the ceiling
    plane leaves no surface just above it, where the 1/r^2 of area sampling
    would blow up."""
    white = s.add_material(Material.diffuse((0.75, 0.75, 0.75)))
    red = s.add_material(Material.diffuse((0.65, 0.05, 0.05)))
    green = s.add_material(Material.diffuse((0.05, 0.65, 0.05)))
    emit = s.add_material(Material.emissive(emitter_radiance))
    c0, c1 = 0.375, 0.625
    s.add_quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1), white)      # floor
    s.add_quad((0, 1, 0), (0, 1, 1), (c0, 1, 1), (c0, 1, 0), white)    # ceiling, left of the opening
    s.add_quad((c1, 1, 0), (c1, 1, 1), (1, 1, 1), (1, 1, 0), white)    # right of it
    s.add_quad((c0, 1, 0), (c0, 1, c0), (c1, 1, c0), (c1, 1, 0), white)  # in front of it
    s.add_quad((c0, 1, c1), (c0, 1, 1), (c1, 1, 1), (c1, 1, c1), white)  # behind it
    s.add_quad((0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1), white)      # back
    s.add_quad((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0), red)        # left
    s.add_quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1), green)      # right
    s.add_quad((c0, 1, c0), (c0, 1, c1), (c1, 1, c1), (c1, 1, c0), emit)
    s.add_light(Light.quad((c0, 1, c0), (0.25, 0, 0), (0, 0, 0.25), emitter_radiance, emit))
    s.background = (0.0, 0.0, 0.0)
    s.ambient = (0.0, 0.0, 0.0)


def box_camera(aspect: float = 1.0) -> CameraArgs:
    return CameraArgs((0.5, 0.5, -1.3), (0.5, 0.45, 0.5), (0, 1, 0), 40.0, aspect)


def mesh_box(subdiv: int = 8, width: int = 1024, height: int = 1024, samples: int = 8,
             depth: int = 12, seed: int = 3) -> Workload:
    s = Scene()
    _box(s)
    mesh_mat = s.add_material(Material.diffuse((0.75, 0.75, 0.75)))
    v, f = icosphere(subdiv)
    disp = value_noise(v, seed)
    v = v * (1.0 + 0.05 * disp)[:, None]
    v = v * 0.35 + np.array([0.5, 0.37, 0.5])
    s.set_mesh(v.astype(np.float32), f.astype(np.int32), mesh_mat)
    s.camera = box_camera(width / height)
    st = RenderSettings(width=width, height=height, samples=samples, max_depth=depth,
                        pathtrace=True, pathtrace_bounces=depth)
    return Workload("mesh_box", s, st)


def adjoint_box(n_spheres: int = 1000, width: int = 512, height: int = 512, samples: int = 4,
                depth: int = 6, seed: int = 5, albedo: np.ndarray | None = None
                ) -> tuple[Workload, np.ndarray, int]:
    """Returns (workload, target albedos (n,3), index of the first sphere
    material). Sphere materials start at the returned index; `albedo` sets
    them (default: the hidden target albedos)."""
    rng = np.random.default_rng(seed)
    target = rng.uniform(0.1, 0.9, size=(n_spheres, 3)).astype(np.float32)
    radii = rng.uniform(0.01, 0.05, size=n_spheres).astype(np.float32)
    centers = (rng.uniform(0.0, 1.0, size=(n_spheres, 3)) * (1.0 - 2 * radii[:, None])
               + radii[:, None]).astype(np.float32)
    centers[:, 1] = np.minimum(centers[:, 1], 0.9)
    s = Scene()
    _box(s)
    alb = target if albedo is None else np.asarray(albedo, np.float32)
    mats = np.zeros(n_spheres, A.MATERIAL_DTYPE)
    mats["kind"] = A.MAT_DIFFUSE
    mats["albedo"] = alb
    mats["ior"] = 1.0
    mats["shininess"] = 32.0
    mats["specular_color"] = 1.0
    first = s.add_material_array(mats)
    s.add_spheres(centers, radii, np.arange(first, first + n_spheres, dtype=np.int32))
    s.camera = box_camera(width / height)
    st = RenderSettings(width=width, height=height, samples=samples, max_depth=depth,
                        pathtrace=True, pathtrace_bounces=depth)
    return Workload("adjoint_box", s, st), target, first
