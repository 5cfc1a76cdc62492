"""Renderer entry point mirroring pencil::Renderer (src/renderer.hpp:155-295).

    settings = RenderSettings(width=320, height=240, samples=2, pathtrace=True,
                              pathtrace_bounces=8)
    r = Renderer(scene, camera, settings)
    pixels = r.render(stats=stats)      # (H, W, 3) float32, row 0 at the top

`render` returns what Renderer::render writes into its std::vector<Color>:
each pixel the mean of its n*n stratified samples. Unlike Pencil's void
render, failures raise GpuError. There is no CPU path: without a CUDA device
the context cannot be created.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .scene import CameraArgs, Scene


@dataclass
class RenderSettings:
    """The fields of pencil::RenderSettings (src/renderer.hpp:34-83) that the
    GPU core implements, plus the GPU engine choices."""
    width: int = 400
    height: int = 300
    samples: int = 4                  # n: n*n samples per pixel
    max_depth: int = 8                # Whitted recursion depth
    shadow_bias: float = 1e-3
    soft_shadow_samples: int = 4
    pathtrace: bool = False
    pathtrace_bounces: int = 4
    # GPU engine
    engine: int = A.ENGINE_WAVEFRONT
    rng: int = A.RNG_COUNTER
    glass: int = A.GLASS_FRESNEL_SPLIT
    seed: int = 0
    sample_offset: int = 0
    count_rays: bool = False
    count_nodes: bool = False
    use_graph: bool = True
    profile_kernels: bool = False
    packets: bool = True           # wavefront: camera rays traced as warp packets
    mis: bool = False              # trace_path_mis's light weights (Pencil's `mis`)
    queue_capacity: int = 0
    sort_key: int = 0
    refill_below: int = 0
    block_size: int = 0            # wavefront threads per block (0: 128)
    binary_tree: bool = False      # megakernel on Pencil's binary tree

    def params(self) -> A.RenderParams:
        p = A.RenderParams()
        p.width, p.height, p.samples = self.width, self.height, self.samples
        p.depth = self.pathtrace_bounces if self.pathtrace else self.max_depth
        p.mode = A.MODE_PATHTRACE if self.pathtrace else A.MODE_WHITTED
        p.engine, p.rng, p.glass = self.engine, self.rng, self.glass
        p.shadow_bias = self.shadow_bias
        p.soft_shadow_samples = self.soft_shadow_samples
        p.seed = self.seed & 0xFFFFFFFF
        p.sample_offset = self.sample_offset
        p.flags = ((A.FLAG_COUNT_RAYS if self.count_rays else 0) |
                   (A.FLAG_COUNT_NODES if self.count_nodes else 0) |
                   (0 if self.use_graph else A.FLAG_NO_GRAPH) |
                   (A.FLAG_PROFILE_KERNELS if self.profile_kernels else 0) |
                   (0 if self.packets else A.FLAG_NO_PACKETS) |
                   (A.FLAG_MIS if self.mis else 0) |
                   (A.FLAG_BINARY_TREE if self.binary_tree else 0))
        p.queue_capacity, p.sort_key = self.queue_capacity, self.sort_key
        p.refill_below = self.refill_below
        p.block_size = self.block_size
        return p


@dataclass
class RenderStats:
    """RenderStats (src/renderer.hpp:85-87) plus the GPU core's counters."""
    rays_traced: int = 0              # Pencil's count: one per trace*/trace_path call
    paths: int = 0
    extension_rays: int = 0
    shadow_rays: int = 0
    node_visits: int = 0
    prim_tests: int = 0
    ext_node_visits: int = 0
    ext_leaf_bytes: int = 0
    shadow_node_visits: int = 0
    shadow_leaf_bytes: int = 0
    device_ms: float = 0.0
    total_ms: float = 0.0
    kernel_ms: dict = field(default_factory=dict)
    kernel_launches: int = 0

    def fill(self, s: A.Stats) -> None:
        self.rays_traced = s.reference_rays
        self.paths, self.extension_rays, self.shadow_rays = s.paths, s.extension_rays, s.shadow_rays
        self.node_visits, self.prim_tests = s.node_visits, s.prim_tests
        self.ext_node_visits, self.ext_leaf_bytes = s.ext_node_visits, s.ext_leaf_bytes
        self.shadow_node_visits, self.shadow_leaf_bytes = s.shadow_node_visits, s.shadow_leaf_bytes
        self.device_ms, self.total_ms = s.device_ms, s.total_ms
        self.kernel_ms = dict(zip(A.KERNEL_CLASSES, list(s.kernel_ms)))
        self.kernel_launches = s.kernel_launches


class GpuContext:
    """One pgpu_ctx: a CUDA device, a stream and the uploaded scenes."""

    def __init__(self, device: int = 0):
        self.lib = A.load()
        h = C.c_void_p()
        rc = self.lib.pgpu_create(device, C.byref(h))
        if rc != A.OK:
            raise A.GpuError(rc, f"pgpu_create(device={device}) failed (no usable CUDA device?)")
        self.h = h

    def close(self) -> None:
        if self.h:
            self.lib.pgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int, what: str) -> None:
        if rc != A.OK:
            msg = self.lib.pgpu_last_error(self.h)
            raise A.GpuError(rc, f"{what}: {msg.decode() if msg else ''}")

    @property
    def stream(self) -> int:
        return self.lib.pgpu_get_stream(self.h) or 0

    def set_stream(self, stream: int | None) -> None:
        self.check(self.lib.pgpu_set_stream(self.h, stream), "pgpu_set_stream")

    def set_timeout(self, ms: int) -> None:
        """Wall-clock budget of a render's device work (0: none)."""
        self.check(self.lib.pgpu_set_timeout(self.h, int(ms)), "pgpu_set_timeout")

    def set_traversal_tree(self, mode: int) -> None:
        """Tree the wide traversals of later uploads walk:
        A.TRAVERSAL_UPLOADED (the uploaded tree, default), A.TRAVERSAL_LBVH
        (a linear BVH over the uploaded leaves, built on the device) or
        A.TRAVERSAL_SAH (a 3-axis binned SAH tree over them, built on the
        device)."""
        self.check(self.lib.pgpu_set_traversal_tree(self.h, int(mode)),
                   "pgpu_set_traversal_tree")

    def upload(self, scene: Scene, nodes: np.ndarray | None = None,
               camera: CameraArgs | None = None) -> int:
        d, keep = scene.desc(nodes, camera)
        sid = C.c_int32(0)
        self.check(self.lib.pgpu_upload_scene(self.h, C.byref(d), C.byref(sid)),
                   "pgpu_upload_scene")
        del keep
        return sid.value

    def free(self, sid: int) -> None:
        self.check(self.lib.pgpu_free_scene(self.h, sid), "pgpu_free_scene")

    def build_bvh_device(self, scene: Scene, method: str = "lbvh") -> tuple[np.ndarray, int]:
        """A BVH built on the GPU, in the node-table format of
        Scene.build_bvh (DFS pre-order): method "lbvh" a linear BVH, "sah"
        Pencil's binned SAH tree. Returns (nodes, depth)."""
        fn = {"lbvh": "pgpu_build_bvh_device", "sah": "pgpu_build_bvh_device_sah"}[method]
        d, keep = scene.desc()
        n = scene.n_unified
        nodes = np.zeros(max(2 * n - 1, 1), A.NODE_DTYPE)
        cnt, depth = C.c_int32(0), C.c_int32(0)
        self.check(getattr(self.lib, fn)(self.h, C.byref(d), A.ptr(nodes), C.byref(cnt),
                                         C.byref(depth)), fn)
        del keep
        return nodes[: cnt.value].copy(), depth.value

    def render_tile(self, sid: int, settings: RenderSettings, x: int, y: int, w: int,
                    h: int) -> np.ndarray:
        """One tile of the distributed worker (render_tile): settings give the
        full image; returns (h, w, 3)."""
        p = settings.params()
        out = np.empty((h, w, 3), np.float32)
        self.check(self.lib.pgpu_render_tile(self.h, sid, C.byref(p), x, y, w, h, A.ptr(out)),
                   "pgpu_render_tile")
        return out

    def scene_info(self, sid: int) -> dict:
        """Sizes of an uploaded scene (device bytes, leaves, binary and wide
        node counts, depth, wide-tree stack need)."""
        info = A.SceneInfo()
        self.check(self.lib.pgpu_get_scene_info(self.h, sid, C.byref(info)),
                   "pgpu_get_scene_info")
        return {name: int(getattr(info, name)) for name, _ in A.SceneInfo._fields_
                if name != "reserved"}

    def tonemap(self, hdr: np.ndarray, tonemap: int = A.TONEMAP_ACES,
                exposure: float = 0.0) -> np.ndarray:
        """Pencil's write_image bytes (exposure, tone curve, gamma 2.2, 8 bits)
        computed on the device from a host HDR image (H, W, 3)."""
        hdr = np.ascontiguousarray(hdr, np.float32)
        out = np.empty(hdr.shape, np.uint8)
        self.check(self.lib.pgpu_tonemap(self.h, A.ptr(hdr), hdr.size // 3, tonemap,
                                         float(exposure), 0, A.ptr(out)), "pgpu_tonemap")
        return out

    def update_materials(self, sid: int, mats: np.ndarray) -> None:
        mats = np.ascontiguousarray(mats, A.MATERIAL_DTYPE)
        self.check(self.lib.pgpu_update_materials(self.h, sid, A.ptr(mats), len(mats)),
                   "pgpu_update_materials")

    def render(self, sid: int, settings: RenderSettings, out: np.ndarray | None = None,
               m2: np.ndarray | None = None, stats: RenderStats | None = None) -> np.ndarray:
        p = settings.params()
        if out is None:
            out = np.empty((settings.height, settings.width, 3), np.float32)
        assert out.dtype == np.float32 and out.size == settings.width * settings.height * 3
        st = A.Stats()
        self.check(self.lib.pgpu_render(self.h, sid, C.byref(p), A.ptr(out), A.ptr(m2),
                                        C.byref(st)), "pgpu_render")
        if stats is not None:
            stats.fill(st)
        return out

    def render_window(self, sid: int, settings: RenderSettings,
                      window: tuple[int, int, int, int], out: np.ndarray | None = None,
                      m2: np.ndarray | None = None,
                      stats: RenderStats | None = None) -> np.ndarray:
        """The window (x, y, w, h) of the image `settings` describe: each
        pixel as in the whole image's render."""
        x, y, w, h = (int(v) for v in window)
        p = settings.params()
        if out is None:
            out = np.empty((h, w, 3), np.float32)
        assert out.dtype == np.float32 and out.size == w * h * 3
        st = A.Stats()
        self.check(self.lib.pgpu_render_window(self.h, sid, C.byref(p), x, y, w, h, A.ptr(out),
                                               A.ptr(m2), C.byref(st)), "pgpu_render_window")
        if stats is not None:
            stats.fill(st)
        return out

    def render_device(self, sid: int, settings: RenderSettings, out_ptr: int,
                      m2_ptr: int | None = None) -> A.Stats:
        """Render into device memory (no host copies)."""
        p = settings.params()
        p.flags |= A.FLAG_DEVICE_OUTPUT
        st = A.Stats()
        self.check(self.lib.pgpu_render(self.h, sid, C.byref(p), out_ptr, m2_ptr, C.byref(st)),
                   "pgpu_render")
        return st

    def render_batch(self, sids: list[int], settings: list[RenderSettings],
                     outs: list[np.ndarray] | None = None, stats: RenderStats | None = None,
                     device_ptrs: list[int] | None = None) -> list[np.ndarray]:
        n = len(sids)
        params = (A.RenderParams * n)(*[s.params() for s in settings])
        if device_ptrs is not None:
            for k in range(n):
                params[k].flags |= A.FLAG_DEVICE_OUTPUT
            ptrs = (C.c_void_p * n)(*device_ptrs)
        else:
            if outs is None:
                outs = [np.empty((s.height, s.width, 3), np.float32) for s in settings]
            ptrs = (C.c_void_p * n)(*[A.ptr(o) for o in outs])
        ids = (C.c_int32 * n)(*sids)
        st = A.Stats()
        self.check(self.lib.pgpu_render_batch(self.h, n, ids, params, ptrs, C.byref(st)),
                   "pgpu_render_batch")
        if stats is not None:
            stats.fill(st)
        return outs

    def trace_rays(self, sid: int, rays: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        n = len(rays)
        prim, t = np.empty(n, np.int32), np.empty(n, np.float32)
        self.check(self.lib.pgpu_trace_rays(self.h, sid, A.ptr(rays), n, A.ptr(prim), A.ptr(t)),
                   "pgpu_trace_rays")
        return prim, t

    def primary_hits(self, sid: int, uv: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
        n = len(uv)
        prim, t = np.empty(n, np.int32), np.empty(n, np.float32)
        self.check(self.lib.pgpu_primary_hits(self.h, sid, A.ptr(uv), n, A.ptr(prim), A.ptr(t)),
                   "pgpu_primary_hits")
        return prim, t

    def adjoint(self, sid: int, settings: RenderSettings, dl_dimage: np.ndarray, n_materials: int,
                n_lights: int, stats: RenderStats | None = None, want_image: bool = False):
        p = settings.params()
        dl = np.ascontiguousarray(dl_dimage, np.float32)
        da = np.zeros((n_materials, 3), np.float64)
        de = np.zeros((n_materials, 3), np.float64)
        dli = np.zeros((max(n_lights, 1), 3), np.float64)
        img = np.empty((settings.height, settings.width, 3), np.float32) if want_image else None
        st = A.Stats()
        self.check(self.lib.pgpu_adjoint(self.h, sid, C.byref(p), A.ptr(dl), A.ptr(da), A.ptr(de),
                                         A.ptr(dli), A.ptr(img), C.byref(st)), "pgpu_adjoint")
        if stats is not None:
            stats.fill(st)
        return da, de, dli[:n_lights], img


_default_ctx: GpuContext | None = None


def default_context() -> GpuContext:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = GpuContext(0)
    return _default_ctx


class Renderer:
    """pencil::Renderer(scene, camera, settings) on the GPU core. The scene is
    uploaded once, at construction (Pencil holds it by reference)."""

    def __init__(self, scene: Scene, camera: CameraArgs | None, settings: RenderSettings,
                 ctx: GpuContext | None = None, nodes: np.ndarray | None = None):
        self.ctx = ctx or default_context()
        self.scene = scene
        self.settings = settings
        self.sid = self.ctx.upload(scene, nodes, camera)

    def render(self, out_pixels: np.ndarray | None = None,
               stats: RenderStats | None = None) -> np.ndarray:
        return self.ctx.render(self.sid, self.settings, out_pixels, None, stats)

    def close(self) -> None:
        if self.sid:
            self.ctx.free(self.sid)
            self.sid = 0
