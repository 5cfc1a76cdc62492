"""ctypes wrapper of the CPU oracle (liboracle.so) and driver of the reference
harness (oracle/_ref/pencil_ref).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker. The GPU core never calls it.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_BIN = HERE / "_ref" / "pencil_ref"

import sys  # noqa: E402

sys.path.insert(0, str(HERE.parent))
from pencil_b200 import _abi as A  # noqa: E402

CNT_REFERENCE_RAYS, CNT_EXTENSION_RAYS, CNT_SHADOW_RAYS, CNT_NODE_VISITS, CNT_PRIM_TESTS = range(5)
(CNT_EXT_NODES, CNT_EXT_PRIMS, CNT_EXT_PRIM_BYTES, CNT_SH_NODES, CNT_SH_PRIMS,
 CNT_SH_PRIM_BYTES, CNT_PRIM_BYTES) = range(5, 12)
CNT_N = 12


class OrcScene(C.Structure):
    _fields_ = [("prims", C.c_void_p), ("n_prims", C.c_int32),
                ("nodes", C.c_void_p), ("n_nodes", C.c_int32),
                ("materials", C.c_void_p), ("n_materials", C.c_int32),
                ("lights", C.c_void_p), ("n_lights", C.c_int32),
                ("cam", C.c_float * 21),
                ("background", C.c_float * 3), ("ambient", C.c_float * 3)]


_lib = None


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    lib.orc_camera_basis.argtypes = [C.POINTER(A.Camera), C.c_void_p]
    lib.orc_render.argtypes = [C.POINTER(OrcScene), C.POINTER(A.RenderParams), C.c_void_p,
                               C.c_void_p, C.c_int32, C.c_void_p]
    lib.orc_render.restype = C.c_int32
    lib.orc_render_split.argtypes = lib.orc_render.argtypes
    lib.orc_render_split.restype = C.c_int32
    for fn in (lib.orc_render_window, lib.orc_render_split_window):
        fn.argtypes = [C.POINTER(OrcScene), C.POINTER(A.RenderParams), C.c_void_p, C.c_void_p,
                       C.c_void_p, C.c_int32, C.c_void_p]
        fn.restype = C.c_int32
    lib.orc_adjoint.argtypes = [C.POINTER(OrcScene), C.POINTER(A.RenderParams), C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
    lib.orc_adjoint.restype = C.c_int32
    lib.orc_trace_rays.argtypes = [C.POINTER(OrcScene), C.c_void_p, C.c_int32, C.c_void_p,
                                   C.c_void_p, C.c_void_p]
    lib.orc_primary_hits.argtypes = [C.POINTER(OrcScene), C.c_void_p, C.c_int32, C.c_void_p,
                                     C.c_void_p]
    lib.orc_camera_rays.argtypes = [C.POINTER(OrcScene), C.c_void_p, C.c_int32, C.c_void_p]
    lib.orc_hit_t_fp64.argtypes = [C.c_void_p, C.c_void_p]
    lib.orc_hit_t_fp64.restype = C.c_double
    lib.orc_rgb8.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_float]
    lib.orc_gamma_monotone.restype = C.c_uint32
    lib.orc_gamma_monotone.argtypes = []
    lib.orc_render_tile.restype = C.c_int32
    lib.orc_render_tile.argtypes = [C.POINTER(OrcScene), C.POINTER(A.RenderParams), C.c_int32,
                                    C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    lib.orc_path_seed.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint32]
    lib.orc_path_seed.restype = C.c_uint32
    _lib = lib
    return lib


class Oracle:
    """A scene prepared for the oracle: unified primitives, Pencil's DFS
    node table (from pgpu_build_bvh or a reference dump) and camera basis."""

    def __init__(self, scene, nodes: np.ndarray | None = None, prims: np.ndarray | None = None):
        self.lib = load()
        self.prims = np.ascontiguousarray(prims if prims is not None else scene.unified_prims())
        if nodes is None:
            nodes, _ = scene.build_bvh()
        self.nodes = np.ascontiguousarray(nodes, A.NODE_DTYPE)
        self.mats = np.ascontiguousarray(scene.material_array())
        self.lights = np.ascontiguousarray(scene.light_array())
        s = OrcScene()
        s.prims, s.n_prims = A.ptr(self.prims), len(self.prims)
        s.nodes, s.n_nodes = A.ptr(self.nodes), len(self.nodes)
        s.materials, s.n_materials = A.ptr(self.mats), len(self.mats)
        s.lights, s.n_lights = A.ptr(self.lights), len(self.lights)
        cam = scene.camera.struct()
        basis = np.zeros(21, np.float32)
        self.lib.orc_camera_basis(C.byref(cam), A.ptr(basis))
        s.cam[:] = basis.tolist()
        s.background[:] = list(map(float, scene.background))
        s.ambient[:] = list(map(float, scene.ambient))
        self.s = s
        self.basis = basis

    def _render(self, fn, settings, threads, want_m2, window):
        p = settings.params()
        x, y, w, h = window if window is not None else (0, 0, settings.width, settings.height)
        out = np.zeros((h, w, 3), np.float32)
        m2 = np.zeros_like(out) if want_m2 else None
        cnt = np.zeros(CNT_N, np.uint64)
        win = np.asarray([x, y, w, h], np.int32)
        rc = fn(C.byref(self.s), C.byref(p), A.ptr(win), A.ptr(out), A.ptr(m2),
                threads or os.cpu_count() or 1, A.ptr(cnt))
        if rc != 0:
            raise ValueError(f"{fn.__name__} rejected its arguments")
        return out, m2, cnt

    def render(self, settings, threads: int | None = None, want_m2: bool = False,
               window: tuple[int, int, int, int] | None = None):
        """The reference algorithm (Pencil's per-pixel RNG, both dielectric
        branches). window = (x, y, w, h): only those pixels of the image."""
        return self._render(self.lib.orc_render_window, settings, threads, want_m2, window)

    def render_split(self, settings, threads: int | None = None, want_m2: bool = False,
                     window: tuple[int, int, int, int] | None = None):
        """The GPU core's production estimator (counter RNG, Fresnel-split
        glass, quad-light NEE) restated on the CPU."""
        return self._render(self.lib.orc_render_split_window, settings, threads, want_m2,
                            window)

    def render_tile(self, settings, x: int, y: int, w: int, h: int) -> np.ndarray:
        """The distributed worker's tile (render_tile) of the full image
        that `settings` describe."""
        p = settings.params()
        out = np.zeros((h, w, 3), np.float32)
        if self.lib.orc_render_tile(C.byref(self.s), C.byref(p), x, y, w, h, A.ptr(out)) != 0:
            raise ValueError("orc_render_tile rejected its arguments")
        return out

    def adjoint(self, settings, dl: np.ndarray, threads: int | None = None):
        """FP64 CPU adjoint of the production estimator: returns
        (d_albedo (n_mat,3), d_emission (n_mat,3), d_light (n_light,3),
        replayed image (H,W,3) float64)."""
        p = settings.params()
        dl = np.ascontiguousarray(dl, np.float32)
        nm, nl = len(self.mats), len(self.lights)
        da, de = np.zeros((nm, 3)), np.zeros((nm, 3))
        dli = np.zeros((max(nl, 1), 3))
        img = np.zeros((settings.height, settings.width, 3))
        rc = self.lib.orc_adjoint(C.byref(self.s), C.byref(p), A.ptr(dl), A.ptr(da), A.ptr(de),
                                  A.ptr(dli), A.ptr(img), threads or os.cpu_count() or 1)
        if rc != 0:
            raise ValueError("orc_adjoint rejected its arguments")
        return da, de, dli[:nl], img

    def trace_rays(self, rays: np.ndarray, counters: bool = False):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        n = len(rays)
        prim, t = np.empty(n, np.int32), np.empty(n, np.float32)
        cnt = np.zeros(CNT_N, np.uint64)
        self.lib.orc_trace_rays(C.byref(self.s), A.ptr(rays), n, A.ptr(prim), A.ptr(t),
                                A.ptr(cnt) if counters else None)
        return (prim, t, cnt) if counters else (prim, t)

    def camera_rays(self, uv: np.ndarray) -> np.ndarray:
        uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
        rays = np.empty((len(uv), 6), np.float32)
        self.lib.orc_camera_rays(C.byref(self.s), A.ptr(uv), len(uv), A.ptr(rays))
        return rays

    def primary_hits(self, uv: np.ndarray):
        uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
        n = len(uv)
        prim, t = np.empty(n, np.int32), np.empty(n, np.float32)
        self.lib.orc_primary_hits(C.byref(self.s), A.ptr(uv), n, A.ptr(prim), A.ptr(t))
        return prim, t

    def hit_t_fp64(self, prim_id: int, ray: np.ndarray) -> float:
        ray = np.ascontiguousarray(ray, np.float32).reshape(6)
        rec = np.ascontiguousarray(self.prims[prim_id:prim_id + 1])
        return self.lib.orc_hit_t_fp64(A.ptr(rec), A.ptr(ray))


def gamma_monotone() -> int:
    """0 when write_image's gamma byte never decreases over the floats of
    [0, 1] with this host's powf (else the bit pattern where it first does)."""
    return int(load().orc_gamma_monotone())


def rgb8(hdr: np.ndarray, tonemap: int = 1, exposure: float = 0.0) -> np.ndarray:
    lib = load()
    hdr = np.ascontiguousarray(hdr, np.float32)
    n = hdr.size // 3
    out = np.empty(hdr.shape[:-1] + (3,), np.uint8)
    lib.orc_rgb8(A.ptr(hdr), n, A.ptr(out), tonemap, exposure)
    return out


def path_seed(i: int, j: int, sample: int, salt: int = 0) -> int:
    return load().orc_path_seed(i, j, sample, salt)


# ---- reference harness ------------------------------------------------------------
def ref_available() -> bool:
    return REF_BIN.exists()


def _run_ref(args: list[str]) -> str:
    proc = subprocess.run([str(REF_BIN)] + args, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"pencil_ref {args[0]} failed: {proc.stderr.strip()}")
    return proc.stdout


def ref_dump(scene) -> tuple[np.ndarray, np.ndarray, int]:
    """The reference's stored primitive state and BVH (DFS) for `scene`."""
    with tempfile.TemporaryDirectory() as d:
        sp, op = Path(d) / "s.bin", Path(d) / "o.bin"
        scene.write(sp)
        _run_ref(["dump", str(sp), str(op)])
        raw = op.read_bytes()
    n_p, n_n, depth = np.frombuffer(raw, np.int32, 3)
    prims = np.frombuffer(raw, A.PRIM_DTYPE, n_p, 12).copy()
    nodes = np.frombuffer(raw, A.NODE_DTYPE, n_n, 12 + 64 * int(n_p)).copy()
    return prims, nodes, int(depth)


def ref_render(scene, width: int, height: int, samples: int, depth: int, pathtrace: bool,
               threads: int = 8, repeat: int = 1, bias: float = 1e-3, soft: int = 4,
               want_image: bool = True, mis: bool = False):
    """Render with the reference's Renderer::render; returns (image, info).
    mis: path tracing with RenderSettings::mis (trace_path_mis)."""
    with tempfile.TemporaryDirectory() as d:
        sp, op = Path(d) / "s.bin", Path(d) / "img.f32"
        scene.write(sp)
        out = _run_ref(["render", str(sp), str(op) if want_image else "-", str(width),
                        str(height), str(samples), str(depth),
                        ("2" if mis else "0") if pathtrace else "1",
                        repr(float(bias)), str(soft), str(threads), str(repeat)])
        info = json.loads(out.strip().splitlines()[-1])
        img = (np.fromfile(op, np.float32).reshape(height, width, 3) if want_image else None)
    return img, info


def ref_hits(scene, rays: np.ndarray):
    with tempfile.TemporaryDirectory() as d:
        sp, rp, op = Path(d) / "s.bin", Path(d) / "r.f32", Path(d) / "o.bin"
        scene.write(sp)
        np.ascontiguousarray(rays, np.float32).tofile(rp)
        _run_ref(["hits", str(sp), str(rp), str(op)])
        raw = np.fromfile(op, np.int32)
    n = len(raw) // 2
    return raw[:n].copy(), raw[n:].view(np.float32).copy()


def ref_tile(scene, width: int, height: int, x: int, y: int, w: int, h: int, samples: int,
             depth: int, bias: float = 1e-3, soft: int = 4) -> np.ndarray:
    """The reference worker's render_tile (src/distributed.hpp:380-434)."""
    with tempfile.TemporaryDirectory() as d:
        sp, op = Path(d) / "s.bin", Path(d) / "tile.f32"
        scene.write(sp)
        _run_ref(["tile", str(sp), str(op), str(width), str(height), str(x), str(y), str(w),
                  str(h), str(samples), str(depth), repr(float(bias)), str(soft)])
        return np.fromfile(op, np.float32).reshape(h, w, 3)


def ref_camrays(scene, uv: np.ndarray) -> np.ndarray:
    with tempfile.TemporaryDirectory() as d:
        sp, up, op = Path(d) / "s.bin", Path(d) / "uv.f32", Path(d) / "o.f32"
        scene.write(sp)
        np.ascontiguousarray(uv, np.float32).tofile(up)
        _run_ref(["camrays", str(sp), str(up), str(op)])
        return np.fromfile(op, np.float32).reshape(-1, 6)


def ref_parse(pecl: str | Path, out_scene: str | Path) -> dict:
    return json.loads(_run_ref(["parse", str(pecl), str(out_scene)]).strip().splitlines()[-1])
