"""ctypes binding of include/pencil_gpu.h (libpencil_gpu.so, built in-tree).

The record types are also exposed as numpy dtypes so that scene tables of
millions of primitives are passed as contiguous arrays without copies.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libpencil_gpu.so"

# status codes
OK = 0
ERR_INVALID_ARG = -1
ERR_UNSUPPORTED = -2
ERR_CUDA = -3
ERR_QUEUE_OVERFLOW = -4
ERR_TIMEOUT = -5
ERR_NO_SCENE = -6
ERR_OUT_OF_MEMORY = -7
ERR_BVH_INVALID = -8

PRIM_SPHERE, PRIM_TRIANGLE, PRIM_CUBE, PRIM_PLANE, PRIM_CYLINDER, PRIM_CONE = range(6)
MAT_DIFFUSE, MAT_METAL, MAT_DIELECTRIC = range(3)
LIGHT_POINT, LIGHT_DIRECTIONAL, LIGHT_QUAD = range(3)
MODE_PATHTRACE, MODE_WHITTED = 0, 1
ENGINE_WAVEFRONT, ENGINE_MEGAKERNEL = 0, 1
RNG_COUNTER, RNG_PIXEL_SEQUENTIAL = 0, 1
GLASS_FRESNEL_SPLIT, GLASS_BOTH_BRANCHES = 0, 1
ABI_VERSION = 2   # PGPU_ABI_VERSION of include/pencil_gpu.h
FLAG_DEVICE_OUTPUT, FLAG_COUNT_RAYS, FLAG_COUNT_NODES, FLAG_NO_GRAPH = 1, 2, 4, 8
FLAG_PROFILE_KERNELS = 16
FLAG_NO_PACKETS = 32
FLAG_MIS = 64
FLAG_BINARY_TREE = 128
TRAVERSAL_UPLOADED, TRAVERSAL_LBVH, TRAVERSAL_SAH = 0, 1, 2
TONEMAP_NONE, TONEMAP_ACES, TONEMAP_REINHARD = 0, 1, 2
TONEMAP_DEVICE_INPUT, TONEMAP_DEVICE_OUTPUT = 1, 2
KERNEL_CLASSES = ("generate", "extend", "shade", "shadow", "accumulate", "megakernel")

PRIM_DTYPE = np.dtype([("type", "<i4"), ("material", "<i4"), ("p", "<f4", (14,))])
NODE_DTYPE = np.dtype([("bmin", "<f4", (3,)), ("left", "<i4"), ("bmax", "<f4", (3,)),
                       ("right", "<i4")])
MATERIAL_DTYPE = np.dtype([("kind", "<i4"), ("albedo", "<f4", (3,)), ("emission", "<f4", (3,)),
                           ("reflectivity", "<f4"), ("ior", "<f4"), ("specular", "<f4"),
                           ("shininess", "<f4"), ("specular_color", "<f4", (3,)),
                           ("flags", "<i4"), ("reserved", "<i4")])
LIGHT_DTYPE = np.dtype([("kind", "<i4"), ("pos", "<f4", (3,)), ("intensity", "<f4", (3,)),
                        ("radius", "<f4"), ("is_emissive", "<i4"), ("edge_u", "<f4", (3,)),
                        ("edge_v", "<f4", (3,)), ("material", "<i4")])
assert PRIM_DTYPE.itemsize == 64 and NODE_DTYPE.itemsize == 32
assert MATERIAL_DTYPE.itemsize == 64 and LIGHT_DTYPE.itemsize == 64


class Camera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("look", C.c_float * 3), ("up", C.c_float * 3),
                ("vfov_deg", C.c_float), ("aspect", C.c_float), ("aperture", C.c_float),
                ("focus_dist", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [("prims", C.c_void_p), ("n_prims", C.c_int32),
                ("mesh_vertices", C.c_void_p), ("n_mesh_vertices", C.c_int32),
                ("mesh_indices", C.c_void_p), ("n_mesh_triangles", C.c_int32),
                ("mesh_materials", C.c_void_p),
                ("nodes", C.c_void_p), ("n_nodes", C.c_int32),
                ("materials", C.c_void_p), ("n_materials", C.c_int32),
                ("lights", C.c_void_p), ("n_lights", C.c_int32),
                ("camera", Camera),
                ("background", C.c_float * 3), ("ambient", C.c_float * 3)]


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("samples", C.c_int32),
                ("depth", C.c_int32), ("mode", C.c_int32), ("engine", C.c_int32),
                ("rng", C.c_int32), ("glass", C.c_int32), ("shadow_bias", C.c_float),
                ("soft_shadow_samples", C.c_int32), ("seed", C.c_uint32),
                ("sample_offset", C.c_int32), ("flags", C.c_int32),
                ("queue_capacity", C.c_int32), ("refill_below", C.c_int32),
                ("sort_key", C.c_int32), ("block_size", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("extension_rays", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("reference_rays", C.c_uint64),
                ("node_visits", C.c_uint64), ("prim_tests", C.c_uint64),
                ("ext_node_visits", C.c_uint64), ("ext_leaf_bytes", C.c_uint64),
                ("shadow_node_visits", C.c_uint64), ("shadow_leaf_bytes", C.c_uint64),
                ("device_ms", C.c_double), ("total_ms", C.c_double),
                ("kernel_ms", C.c_double * 6),
                ("kernel_launches", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("reserved", "kernel_ms")}
        d["kernel_ms"] = dict(zip(KERNEL_CLASSES, list(self.kernel_ms)))
        return d


class SceneInfo(C.Structure):
    _fields_ = [("device_bytes", C.c_int64), ("n_leaves", C.c_int32),
                ("n_interior", C.c_int32), ("n_wide", C.c_int32), ("bvh_depth", C.c_int32),
                ("wide_stack", C.c_int32), ("wide_width", C.c_int32)]


EXPORTS = {
    "pgpu_abi_version": (C.c_int32, []),
    "pgpu_create": (C.c_int32, [C.c_int32, C.POINTER(C.c_void_p)]),
    "pgpu_destroy": (None, [C.c_void_p]),
    "pgpu_last_error": (C.c_char_p, [C.c_void_p]),
    "pgpu_set_stream": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "pgpu_get_stream": (C.c_void_p, [C.c_void_p]),
    "pgpu_set_timeout": (C.c_int32, [C.c_void_p, C.c_int32]),
    "pgpu_set_traversal_tree": (C.c_int32, [C.c_void_p, C.c_int32]),
    "pgpu_make_prim": (C.c_int32, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_float, C.c_float, C.c_void_p]),
    "pgpu_build_bvh": (C.c_int32, [C.POINTER(SceneDesc), C.c_void_p, C.POINTER(C.c_int32),
                                   C.POINTER(C.c_int32)]),
    "pgpu_upload_scene": (C.c_int32, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(C.c_int32)]),
    "pgpu_free_scene": (C.c_int32, [C.c_void_p, C.c_int32]),
    "pgpu_render": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(RenderParams), C.c_void_p,
                                C.c_void_p, C.POINTER(Stats)]),
    "pgpu_render_window": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(RenderParams),
                                       C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                       C.c_void_p, C.POINTER(Stats)]),
    "pgpu_render_batch": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.POINTER(Stats)]),
    "pgpu_trace_rays": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                    C.c_void_p]),
    "pgpu_primary_hits": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                      C.c_void_p]),
    "pgpu_adjoint": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(RenderParams), C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.POINTER(Stats)]),
    "pgpu_update_materials": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]),
    "pgpu_get_scene_info": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(SceneInfo)]),
    "pgpu_tonemap": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_float,
                                 C.c_int32, C.c_void_p]),
    "pgpu_render_tile": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(RenderParams), C.c_int32,
                                     C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    "pgpu_build_bvh_device": (C.c_int32, [C.c_void_p, C.POINTER(SceneDesc), C.c_void_p,
                                          C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "pgpu_build_bvh_device_sah": (C.c_int32, [C.c_void_p, C.POINTER(SceneDesc), C.c_void_p,
                                          C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "pgpu_render_noalloc": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(RenderParams),
                                        C.c_void_p, C.c_void_p]),
}

_lib: C.CDLL | None = None


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load libpencil_gpu.so, compiling it first if it is absent (nvcc is
    required; there is no CPU implementation to fall back to)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists() or os.environ.get("PGPU_REBUILD") == "1":
        if not build_if_missing:
            raise RuntimeError(f"{LIB_PATH} is missing; run pencil_b200/build.py")
        from . import build as _build
        _build.build()
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.pgpu_abi_version() != ABI_VERSION:
        raise RuntimeError("libpencil_gpu.so ABI version mismatch")
    _lib = lib
    return lib


class GpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pencil_gpu error {code}: {msg}")
        self.code = code


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C-ABI must be contiguous"
    return a.ctypes.data
