"""pgpu_render_noalloc: rendering without allocating device memory.

Callers whose device memory belongs to someone else (a framework's caching
allocator), or who cannot afford the device-wide synchronisation of
cudaMalloc/cudaFree in the middle of a frame, render through this entry
point: the wavefront kernels run over a fixed-size array compiled into the
library, on a scene uploaded beforehand, into output buffers the caller
owns. Its images must equal those of pgpu_render with the wavefront engine,
call after call, since every call reuses (and must clean up) the same array.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from pencil_b200 import _abi as A
from pencil_b200 import workloads as W
from pencil_b200.renderer import RenderSettings

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def noalloc(gpu, sid, st, out, m2=None) -> int:
    p = st.params()
    p.flags |= A.FLAG_DEVICE_OUTPUT
    return gpu.lib.pgpu_render_noalloc(gpu.h, sid, C.byref(p), out.data_ptr(),
                                       m2.data_ptr() if m2 is not None else None)


def case(name):
    if name == "mesh_box_quad":
        w = W.mesh_box(subdiv=2, width=40, height=40, samples=4, depth=6)
        return w.scene, None, w.settings
    scene, fx = load_golden(name)
    wd, ht, _, depth = (int(x) for x in fx["settings"])
    st = RenderSettings(width=wd, height=ht, samples=8, max_depth=depth, pathtrace=True,
                        pathtrace_bounces=depth)
    return scene, fx["nodes"], st


@pytest.mark.parametrize("name,pathtrace", [("c1", True), ("cloud2k", True), ("cornell_box", True),
                                            ("cornell_box", False), ("mesh_box_quad", True),
                                            ("c1", False)])
def test_noalloc_equals_render_on_two_calls_in_a_row(gpu, name, pathtrace):
    scene, nodes, st = case(name)
    st.pathtrace = pathtrace
    sid = gpu.upload(scene, nodes)
    ref = gpu.render(sid, st)                       # the existing entry point
    m2_ref = np.zeros_like(ref)
    gpu.render(sid, st, m2=m2_ref)
    out = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
    m2 = torch.empty_like(out)
    for _ in range(2):
        out.fill_(float("nan"))
        m2.fill_(float("nan"))
        torch.cuda.synchronize()
        gpu.check(noalloc(gpu, sid, st, out, m2), "pgpu_render_noalloc")
        got, got2 = out.cpu().numpy(), m2.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
        assert np.array_equal(got2.view(np.uint32), m2_ref.view(np.uint32))
    gpu.free(sid)


@pytest.mark.parametrize("name,samples", [("cornell_box", 3), ("cloud2k", 2)])
def test_noalloc_several_chunks_equal_render(gpu, name, samples):
    """More paths than the 65,536 the array holds at once, so the render runs
    chunk after chunk and the last chunk is partial: 128x96 pixels at 9
    samples are 110,592 paths (chunks of 7,281 and 5,007 pixels); 192x128 at
    4 samples are 98,304 paths (16,384 and 8,192 pixels). Each chunk must
    restart its queues and cursors and accumulate into its own pixels; the
    image equals pgpu_render's bit for bit, twice in a row."""
    scene, nodes, st = case(name)
    st.width, st.height, st.samples = 128, 96, samples
    if samples == 2:
        st.width, st.height = 192, 128
    assert st.width * st.height * samples * samples > 65536
    sid = gpu.upload(scene, nodes)
    ref = gpu.render(sid, st)
    m2_ref = np.zeros_like(ref)
    gpu.render(sid, st, m2=m2_ref)
    out = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
    m2 = torch.empty_like(out)
    for _ in range(2):
        out.fill_(float("nan"))
        m2.fill_(float("nan"))
        torch.cuda.synchronize()
        gpu.check(noalloc(gpu, sid, st, out, m2), "pgpu_render_noalloc")
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))
        assert np.array_equal(m2.cpu().numpy().view(np.uint32), m2_ref.view(np.uint32))
    gpu.free(sid)


def test_noalloc_allocates_nothing(gpu):
    scene, nodes, st = case("cloud2k")
    sid = gpu.upload(scene, nodes)
    out = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
    gpu.check(noalloc(gpu, sid, st, out), "first call (set-up)")
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        gpu.check(noalloc(gpu, sid, st, out), "pgpu_render_noalloc")
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == before
    gpu.free(sid)


def test_noalloc_rejects_work_beyond_its_capacity(gpu):
    # glass makes Whitted vertices: 4 + 1 + 1 + 4 soft-shadow rays at each
    scene, nodes, st = case("prims_mix")
    sid = gpu.upload(scene, nodes)
    out = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
    for pathtrace in (True, False):
        st.pathtrace = pathtrace
        assert noalloc(gpu, sid, st, out) == A.ERR_INVALID_ARG
        assert b"4 shadow rays" in gpu.lib.pgpu_last_error(gpu.h)
    gpu.free(sid)
    scene, nodes, st = case("cornell_box")
    sid = gpu.upload(scene, nodes)
    out = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
    st.pathtrace_bounces = 65
    assert noalloc(gpu, sid, st, out) == A.ERR_INVALID_ARG
    st.pathtrace_bounces = 6
    st.sort_key = 1
    assert noalloc(gpu, sid, st, out) == A.ERR_INVALID_ARG
    st.sort_key = 0
    gpu.check(noalloc(gpu, sid, st, out), "within limits")
    gpu.free(sid)
