"""Scene description on the host, mirroring Pencil's types.

Pencil keeps its Scene/Material/Light/Camera classes (src/scene.hpp,
src/material.hpp, src/light.hpp, src/camera.hpp); a Pencil build hands them to
the GPU core through include/pencil_gpu.h. This module is the same data in
Python, for callers that build scenes programmatically (the benchmark
workloads, the tests): materials and lights with Pencil's factory semantics
(make_diffuse / make_metal / make_dielectric / make_emissive,
make_point_light / make_directional_light), primitives in their stored
post-constructor state, an optional indexed triangle mesh, and the camera's
constructor arguments.
"""
from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass, field
from pathlib import Path
from typing import Sequence

import numpy as np

from . import _abi as A


def _f3(v) -> np.ndarray:
    a = np.asarray(v, dtype=np.float32).reshape(3)
    return a


def normalized(v) -> np.ndarray:
    """Vec3::normalized in float32 (src/vec3.hpp:64-69): sqrt((x*x + y*y) + z*z),
    each component divided by it, zero if the length is <= 1e-12."""
    x, y, z = (np.float32(c) for c in _f3(v))
    ln = np.sqrt(np.float32(np.float32(x * x + y * y) + z * z), dtype=np.float32)
    if not ln > np.float32(1e-12):
        return np.zeros(3, np.float32)
    return np.array([x / ln, y / ln, z / ln], dtype=np.float32)


@dataclass
class Material:
    """src/material.hpp:29-80, the fields the GPU core supports."""
    kind: int = A.MAT_DIFFUSE
    albedo: Sequence[float] = (0.8, 0.8, 0.8)
    emission: Sequence[float] = (0.0, 0.0, 0.0)
    reflectivity: float = 0.0
    ior: float = 1.0
    specular: float = 0.0
    shininess: float = 32.0
    specular_color: Sequence[float] = (1.0, 1.0, 1.0)

    @staticmethod
    def diffuse(albedo, spec: float = 0.0, shininess: float = 32.0,
                spec_color=(1.0, 1.0, 1.0)) -> "Material":   # make_diffuse
        return Material(A.MAT_DIFFUSE, tuple(albedo), (0, 0, 0), 0.0, 1.0, spec, shininess,
                        tuple(spec_color))

    @staticmethod
    def metal(albedo, fuzz: float = 0.0) -> "Material":      # make_metal
        f = min(max(float(fuzz), 0.0), 1.0)
        return Material(A.MAT_METAL, tuple(albedo), (0, 0, 0),
                        float(np.float32(1.0) - np.float32(f)), 1.0, 0.0)

    @staticmethod
    def dielectric(ior: float, tint=(1.0, 1.0, 1.0)) -> "Material":   # make_dielectric
        return Material(A.MAT_DIELECTRIC, tuple(tint), (0, 0, 0), 0.0, ior, 0.0)

    @staticmethod
    def emissive(emit) -> "Material":                        # make_emissive
        return Material(A.MAT_DIFFUSE, (0.0, 0.0, 0.0), tuple(emit))

    def record(self) -> np.void:
        r = np.zeros((), A.MATERIAL_DTYPE)
        r["kind"] = self.kind
        r["albedo"] = self.albedo
        r["emission"] = self.emission
        r["reflectivity"] = self.reflectivity
        r["ior"] = self.ior
        r["specular"] = self.specular
        r["shininess"] = self.shininess
        r["specular_color"] = self.specular_color
        return r


@dataclass
class Light:
    """src/light.hpp:15-46, plus rectangular area lights for NEE."""
    kind: int = A.LIGHT_POINT
    pos: Sequence[float] = (0.0, 5.0, 0.0)
    intensity: Sequence[float] = (1.0, 1.0, 1.0)
    radius: float = 0.0
    is_emissive: bool = False
    edge_u: Sequence[float] = (0.0, 0.0, 0.0)
    edge_v: Sequence[float] = (0.0, 0.0, 0.0)
    material: int = 0

    @staticmethod
    def point(pos, intensity, radius: float = 0.0, is_emissive: bool = False) -> "Light":
        return Light(A.LIGHT_POINT, tuple(pos), tuple(intensity), radius, is_emissive)

    @staticmethod
    def directional(direction, intensity) -> "Light":
        return Light(A.LIGHT_DIRECTIONAL, tuple(normalized(direction)), tuple(intensity), 0.0)

    @staticmethod
    def quad(corner, edge_u, edge_v, radiance, material: int) -> "Light":
        return Light(A.LIGHT_QUAD, tuple(corner), tuple(radiance), 0.0, False, tuple(edge_u),
                     tuple(edge_v), material)

    def record(self) -> np.void:
        r = np.zeros((), A.LIGHT_DTYPE)
        r["kind"] = self.kind
        r["pos"] = self.pos
        r["intensity"] = self.intensity
        r["radius"] = self.radius
        r["is_emissive"] = int(self.is_emissive)
        r["edge_u"] = self.edge_u
        r["edge_v"] = self.edge_v
        r["material"] = self.material
        return r


@dataclass
class CameraArgs:
    """Camera constructor arguments (src/camera.hpp:29-36)."""
    eye: Sequence[float] = (0.0, 1.5, -5.0)
    look: Sequence[float] = (0.0, 0.0, 0.0)
    up: Sequence[float] = (0.0, 1.0, 0.0)
    vfov_deg: float = 60.0
    aspect: float = 4.0 / 3.0
    aperture: float = 0.0
    focus_dist: float = 1.0

    def struct(self) -> A.Camera:
        c = A.Camera()
        c.eye[:] = list(map(float, self.eye))
        c.look[:] = list(map(float, self.look))
        c.up[:] = list(map(float, self.up))
        c.vfov_deg, c.aspect = self.vfov_deg, self.aspect
        c.aperture, c.focus_dist = self.aperture, self.focus_dist
        return c


def make_prim(ptype: int, material: int, a=None, b=None, c=None, s0: float = 0.0,
              s1: float = 0.0) -> np.ndarray:
    """A primitive's stored state from its constructor arguments (the C
    library's pgpu_make_prim, which repeats the constructors' arithmetic)."""
    lib = A.load()
    out = np.zeros(1, A.PRIM_DTYPE)
    args = [None if v is None else np.ascontiguousarray(_f3(v)) for v in (a, b, c)]
    rc = lib.pgpu_make_prim(ptype, material, *[A.ptr(v) for v in args], s0, s1, A.ptr(out))
    if rc != A.OK:
        raise A.GpuError(rc, "pgpu_make_prim: invalid primitive")
    return out


class Scene:
    """Primitive list, materials, lights, camera, background and ambient
    (src/scene.hpp:21-105). Primitive indices are assigned in add order; mesh
    triangles follow the explicit primitives in the unified index space."""

    def __init__(self):
        self._mat_chunks: list[np.ndarray] = []
        self.lights: list[Light] = []
        self._chunks: list[np.ndarray] = []
        self._prims: np.ndarray | None = None
        self.mesh_vertices = np.zeros((0, 3), np.float32)
        self.mesh_indices = np.zeros((0, 3), np.int32)
        self.mesh_materials = np.zeros((0,), np.int32)
        self.camera = CameraArgs()
        self.background = (0.05, 0.06, 0.09)      # Scene::background default
        self.ambient = (0.06, 0.06, 0.08)         # Scene::ambient default

    # ---- building ------------------------------------------------------
    def add_material(self, m: Material) -> int:
        self._mat_chunks.append(np.asarray(m.record()).reshape(1))
        return self.n_materials - 1

    def add_material_array(self, recs: np.ndarray) -> int:
        """Append material records (MATERIAL_DTYPE); returns the first id."""
        first = self.n_materials
        self._mat_chunks.append(np.ascontiguousarray(recs, A.MATERIAL_DTYPE))
        return first

    @property
    def n_materials(self) -> int:
        return sum(len(c) for c in self._mat_chunks)

    def add_light(self, l: Light) -> int:
        self.lights.append(l)
        return len(self.lights) - 1

    def _add(self, rec: np.ndarray) -> int:
        self._chunks.append(rec)
        self._prims = None
        return self.n_prims - 1

    def add_sphere(self, center, radius: float, material: int) -> int:
        return self._add(make_prim(A.PRIM_SPHERE, material, center, s0=radius))

    def add_spheres(self, centers: np.ndarray, radii: np.ndarray, materials: np.ndarray) -> None:
        n = len(radii)
        rec = np.zeros(n, A.PRIM_DTYPE)
        rec["type"] = A.PRIM_SPHERE
        rec["material"] = materials
        rec["p"][:, :3] = np.asarray(centers, np.float32)
        rec["p"][:, 3] = np.asarray(radii, np.float32)
        self._add(rec)

    def add_triangle(self, a, b, c, material: int) -> int:
        return self._add(make_prim(A.PRIM_TRIANGLE, material, a, b, c))

    def add_quad(self, a, b, c, d, material: int) -> None:
        """make_quad (src/primitives.hpp:390-396): triangles (a,b,c), (a,c,d)."""
        self.add_triangle(a, b, c, material)
        self.add_triangle(a, c, d, material)

    def add_cube(self, center, half: float, material: int) -> int:
        return self._add(make_prim(A.PRIM_CUBE, material, center, s0=half))

    def add_plane(self, point, normal, material: int) -> int:
        return self._add(make_prim(A.PRIM_PLANE, material, point, normal))

    def add_cylinder(self, center, axis, radius: float, height: float, material: int) -> int:
        return self._add(make_prim(A.PRIM_CYLINDER, material, center, axis, s0=radius, s1=height))

    def add_cone(self, apex, axis, radius: float, height: float, material: int) -> int:
        return self._add(make_prim(A.PRIM_CONE, material, apex, axis, s0=radius, s1=height))

    def add_prims(self, recs: np.ndarray) -> None:
        self._add(np.ascontiguousarray(recs, A.PRIM_DTYPE))

    def set_mesh(self, vertices: np.ndarray, indices: np.ndarray, materials) -> None:
        self.mesh_vertices = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        self.mesh_indices = np.ascontiguousarray(indices, np.int32).reshape(-1, 3)
        m = np.asarray(materials, np.int32)
        if m.ndim == 0:
            m = np.full(len(self.mesh_indices), int(m), np.int32)
        self.mesh_materials = np.ascontiguousarray(m)

    # ---- views ---------------------------------------------------------
    @property
    def prims(self) -> np.ndarray:
        if self._prims is None:
            self._prims = (np.concatenate(self._chunks) if self._chunks
                           else np.zeros(0, A.PRIM_DTYPE))
            self._chunks = [self._prims] if len(self._prims) else []
        return self._prims

    @property
    def n_prims(self) -> int:
        return sum(len(c) for c in self._chunks)

    @property
    def n_unified(self) -> int:
        return self.n_prims + len(self.mesh_indices)

    def material_array(self) -> np.ndarray:
        if len(self._mat_chunks) != 1:
            arr = (np.concatenate(self._mat_chunks) if self._mat_chunks
                   else np.zeros(0, A.MATERIAL_DTYPE))
            self._mat_chunks = [arr] if len(arr) else []
        return self._mat_chunks[0] if self._mat_chunks else np.zeros(0, A.MATERIAL_DTYPE)

    def set_material_array(self, recs: np.ndarray) -> None:
        """Replace every material (same count expected by uploaded scenes)."""
        self._mat_chunks = [np.ascontiguousarray(recs, A.MATERIAL_DTYPE).copy()]

    def light_array(self) -> np.ndarray:
        out = np.zeros(len(self.lights), A.LIGHT_DTYPE)
        for k, l in enumerate(self.lights):
            out[k] = l.record()
        return out

    def unified_prims(self) -> np.ndarray:
        """Explicit primitives followed by the mesh triangles as triangle
        records (the index space of BVH leaves)."""
        prims = self.prims
        nt = len(self.mesh_indices)
        if nt == 0:
            return prims.copy()
        tri = np.zeros(nt, A.PRIM_DTYPE)
        tri["type"] = A.PRIM_TRIANGLE
        tri["material"] = self.mesh_materials
        tri["p"][:, :9] = self.mesh_vertices[self.mesh_indices].reshape(nt, 9)
        return np.concatenate([prims, tri])

    def desc(self, nodes: np.ndarray | None = None, camera: CameraArgs | None = None):
        """pgpu_scene for this scene; returns (struct, keepalive)."""
        keep = [self.prims, self.mesh_vertices, self.mesh_indices, self.mesh_materials,
                self.material_array(), self.light_array()]
        d = A.SceneDesc()
        d.prims, d.n_prims = A.ptr(keep[0]), len(keep[0])
        d.mesh_vertices, d.n_mesh_vertices = A.ptr(keep[1]), len(keep[1])
        d.mesh_indices, d.n_mesh_triangles = A.ptr(keep[2]), len(keep[2])
        d.mesh_materials = A.ptr(keep[3])
        d.materials, d.n_materials = A.ptr(keep[4]), len(keep[4])
        d.lights, d.n_lights = A.ptr(keep[5]), len(keep[5])
        if nodes is not None:
            nodes = np.ascontiguousarray(nodes, A.NODE_DTYPE)
            keep.append(nodes)
            d.nodes, d.n_nodes = A.ptr(nodes), len(nodes)
        d.camera = (camera or self.camera).struct()
        d.background[:] = list(map(float, self.background))
        d.ambient[:] = list(map(float, self.ambient))
        return d, keep

    def build_bvh(self) -> tuple[np.ndarray, int]:
        """Pencil's SAH BVH (src/bvh.hpp:54-192) in DFS pre-order, built by the
        C library; returns (nodes, depth)."""
        lib = A.load()
        d, keep = self.desc()
        n = self.n_unified
        nodes = np.zeros(max(2 * n - 1, 1), A.NODE_DTYPE)
        cnt, depth = C.c_int32(0), C.c_int32(0)
        rc = lib.pgpu_build_bvh(C.byref(d), A.ptr(nodes), C.byref(cnt), C.byref(depth))
        if rc != A.OK:
            raise A.GpuError(rc, "pgpu_build_bvh failed")
        return nodes[: cnt.value].copy(), depth.value

    # ---- scene files (exchange format of the reference harness) ----------
    MAGIC = b"PGPUSCN1"

    def write(self, path: str | Path) -> None:
        prims = self.unified_prims()
        mats, lights = self.material_array(), self.light_array()
        cam = self.camera
        with open(path, "wb") as f:
            f.write(self.MAGIC)
            f.write(struct.pack("<3i", len(prims), len(mats), len(lights)))
            f.write(np.array(list(cam.eye) + list(cam.look) + list(cam.up) +
                             [cam.vfov_deg, cam.aspect, cam.aperture, cam.focus_dist],
                             np.float32).tobytes())
            f.write(np.array(list(self.background) + list(self.ambient), np.float32).tobytes())
            f.write(prims.tobytes())
            f.write(mats.tobytes())
            f.write(lights.tobytes())

    @classmethod
    def read(cls, path: str | Path) -> "Scene":
        raw = Path(path).read_bytes()
        if raw[:8] != cls.MAGIC:
            raise ValueError(f"{path}: not a scene file")
        n_p, n_m, n_l = struct.unpack_from("<3i", raw, 8)
        off = 20
        cam = np.frombuffer(raw, np.float32, 13, off); off += 52
        bgamb = np.frombuffer(raw, np.float32, 6, off); off += 24
        prims = np.frombuffer(raw, A.PRIM_DTYPE, n_p, off).copy(); off += 64 * n_p
        mats = np.frombuffer(raw, A.MATERIAL_DTYPE, n_m, off).copy(); off += 64 * n_m
        lights = np.frombuffer(raw, A.LIGHT_DTYPE, n_l, off).copy()
        s = cls()
        s.add_prims(prims)
        s.add_material_array(mats)
        for l in lights:
            s.add_light(Light(int(l["kind"]), tuple(l["pos"]), tuple(l["intensity"]),
                              float(l["radius"]), bool(l["is_emissive"]), tuple(l["edge_u"]),
                              tuple(l["edge_v"]), int(l["material"])))
        s.camera = CameraArgs(tuple(cam[0:3]), tuple(cam[3:6]), tuple(cam[6:9]), float(cam[9]),
                              float(cam[10]), float(cam[11]), float(cam[12]))
        s.background = tuple(float(x) for x in bgamb[:3])
        s.ambient = tuple(float(x) for x in bgamb[3:])
        return s
