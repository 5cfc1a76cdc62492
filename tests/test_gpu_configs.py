"""The GPU core on the benchmark configurations at their configured sizes.

Every comparison goes through the oracle, which reproduces the reference
renderer bit for bit on these very scenes and sizes
(test_oracle_config_pins.py, against digests of the reference's output):

  C1  three spheres, 320x240, n=2, depth 8: the megakernel in Pencil's exact
      mode (per-pixel RNG, both dielectric branches) against the reference
      image; the production estimator (counter RNG, Fresnel-split glass)
      within 3 sigma of the reference expectation at n=8.
  C2  100k spheres, the full 1280x720 frame, n=4, depth 8: the wavefront
      against the reference expectation within 3 sigma (4x4-pixel blocks of
      256 samples each), and path for path against the oracle's restatement
      of the production estimator on a window of the frame.
  C3  the full 1,310,720-triangle mesh box, 1024x1024, depth 12: the
      wavefront with quad-light NEE path for path against the oracle's
      restatement on windows of the frame (n=2), and within 3 sigma of the
      reference's BSDF-only expectation at the configured n=8 (4x4 blocks).
  C4  32 scenes of the batch workload at their drawn sizes: one batched
      launch sequence equals the scenes rendered one at a time, bit for bit.
  (C5, the adjoint box at 512x512, is in test_gpu_adjoint.py.)

And Pencil's own golden PNGs (Whitted mode, the CLI default) through the
GPU: exact-mode render at the golden size, device tone map, bytes against
the oracle's bytes, which equal the reference's PNG bytes.
"""
from __future__ import annotations

import dataclasses
import hashlib

import numpy as np
import pytest

from conftest import load_golden, png_goldens
from oracle import oracle as O
from pencil_b200 import _abi as A
from pencil_b200 import workloads as W
from pencil_b200.renderer import RenderSettings

pytestmark = pytest.mark.gpu


def near_exact(img, ref, frac=0.005):
    """Equal up to the last bits of libm's cos/sin/pow, which can flip a
    branch of a few paths: at most `frac` of channels beyond 1e-4 relative."""
    rel = np.abs(img.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-3)
    assert np.isfinite(img).all()
    bad = (rel > 1e-4).mean()
    assert bad <= frac, f"{bad:.5f} of channels differ"
    assert abs(img.mean() - ref.mean()) <= 1e-4 * max(abs(ref.mean()), 1e-3)
    return bad


def block_z(mu_a, m2_a, mu_b, m2_b, n, b):
    """z-scores of b x b pixel-block sums of two independent estimates with
    n samples per pixel each (per-pixel variances from the second moments)."""
    H, W_ = mu_a.shape[:2]
    H, W_ = H - H % b, W_ - W_ % b

    def blk(x):
        x = x[:H, :W_].astype(np.float64)
        return x.reshape(H // b, b, W_ // b, b, 3).sum(axis=(1, 3))

    va = np.maximum(m2_a.astype(np.float64) - mu_a.astype(np.float64) ** 2, 0) * n / (n - 1)
    vb = np.maximum(m2_b.astype(np.float64) - mu_b.astype(np.float64) ** 2, 0) * n / (n - 1)
    diff = blk(mu_a) - blk(mu_b)
    se = np.sqrt(blk(va) / n + blk(vb) / n)
    tol = 1e-5 * np.maximum(np.abs(blk(mu_b)), 1e-3)
    z = np.where(se > 0, diff / np.maximum(se, 1e-30), np.where(np.abs(diff) <= tol, 0.0, np.inf))
    return z, diff, se


def test_c1_exact_mode_equals_reference_at_full_size(gpu):
    w = W.three_spheres_pt(320, 240, 2, 8)
    sid = gpu.upload(w.scene)
    ref, _, _ = O.Oracle(w.scene).render(w.settings)
    for binary in (True, False):
        st = dataclasses.replace(w.settings, engine=A.ENGINE_MEGAKERNEL,
                                 rng=A.RNG_PIXEL_SEQUENTIAL, glass=A.GLASS_BOTH_BRANCHES,
                                 binary_tree=binary)
        near_exact(gpu.render(sid, st), ref)
    gpu.free(sid)


def test_c1_production_estimator_three_sigma_at_full_size(gpu):
    w = W.three_spheres_pt(320, 240, 8, 8)
    sid = gpu.upload(w.scene)
    mu_o, m2_o, _ = O.Oracle(w.scene).render(w.settings, want_m2=True)
    m2_g = np.zeros_like(mu_o)
    mu_g = gpu.render(sid, w.settings, m2=m2_g)
    z, diff, se = block_z(mu_g, m2_g, mu_o, m2_o, 64, 1)
    frac = (np.abs(z) > 3).mean()
    assert frac <= 0.015, f"{frac:.4f} of channels beyond 3 sigma"
    assert abs(diff.sum()) <= 3 * np.sqrt((se ** 2).sum())
    gpu.free(sid)


@pytest.fixture(scope="module")
def cloud(gpu):
    w = W.sphere_cloud()
    sid = gpu.upload(w.scene)
    yield w, sid
    gpu.free(sid)


def test_c2_full_frame_three_sigma_against_reference(gpu, cloud):
    """The full 1280x720 frame at 16 spp, depth 8 (14.7M paths on each
    side): the reference algorithm's expectation (the oracle in its
    bit-exact mode, which takes most of this test's time) against the GPU
    wavefront's production estimator."""
    w, sid = cloud
    st = dataclasses.replace(w.settings, engine=A.ENGINE_WAVEFRONT)
    mu_o, m2_o, _ = O.Oracle(w.scene).render(st, want_m2=True)
    m2_g = np.zeros_like(mu_o)
    mu_g = gpu.render(sid, st, m2=m2_g)
    assert np.isfinite(mu_g).all() and (mu_g >= 0).all()
    z, diff, se = block_z(mu_g, m2_g, mu_o, m2_o, 16, 4)
    frac = (np.abs(z) > 3).mean()
    print(f"C2 full frame: {frac:.5f} of 4x4-block channels beyond 3 sigma; "
          f"image mean {mu_g.mean():.6f} (reference {mu_o.mean():.6f})")
    assert frac <= 0.015, f"{frac:.4f} of block channels beyond 3 sigma"
    assert abs(diff.sum()) <= 3 * np.sqrt((se ** 2).sum())


@pytest.mark.parametrize("window", [(560, 300, 160, 120), (0, 0, 96, 64)])
def test_c2_full_frame_path_for_path_on_windows(gpu, cloud, window):
    """The full frame, 16 spp, against the oracle's restatement of the
    production estimator on windows of it. Path for path at depth 1 (camera
    rays, hits, shadow rays). From the first scattered bounce on, the
    device's cosf/sinf and the host libm's differ in the last bit now and
    then; in the dense middle of the cloud such a direction can graze a
    different sphere, and from there the path is another (equally valid)
    sample: at depth 2 about 1.5% of the middle window's pixel channels hold
    such a path, at depth 8 about a fifth. There the two images are compared
    as estimates of the same expectation (3 sigma per channel and for the
    window's mean; most samples are shared, so the test is conservative)."""
    w, sid = cloud
    x, y, ww, wh = window
    orc = O.Oracle(w.scene)
    for engine in (A.ENGINE_WAVEFRONT, A.ENGINE_MEGAKERNEL):
        st = dataclasses.replace(w.settings, engine=engine, pathtrace_bounces=1, max_depth=1)
        img = gpu.render_window(sid, st, window)
        ref, _, _ = orc.render_split(st, window=window)
        near_exact(img, ref)
        for depth in (2, 8):
            st = dataclasses.replace(w.settings, engine=engine, pathtrace_bounces=depth,
                                     max_depth=depth)
            m2_g = np.zeros((wh, ww, 3), np.float32)
            mu_g = gpu.render_window(sid, st, window, m2=m2_g)
            mu_o, m2_o, _ = orc.render_split(st, window=window, want_m2=True)
            same = np.all(mu_g.view(np.uint32) == mu_o.view(np.uint32), axis=2).mean()
            z, diff, se = block_z(mu_g, m2_g, mu_o, m2_o, 16, 1)
            print(f"C2 window {window} engine {engine}: depth {depth}, {same:.4f} of pixels "
                  f"bit-equal; {(np.abs(z) > 3).mean():.4f} of channels beyond 3 sigma")
            assert same >= 0.5
            assert (np.abs(z) > 3).mean() <= 0.015
            assert abs(diff.sum()) <= 3 * np.sqrt((se ** 2).sum())


@pytest.fixture(scope="module")
def mesh(gpu):
    w = W.mesh_box()
    nodes, _ = w.scene.build_bvh()
    sid = gpu.upload(w.scene, nodes)
    yield w, sid, O.Oracle(w.scene, nodes)
    gpu.free(sid)


@pytest.mark.parametrize("window", [(400, 320, 128, 96), (96, 640, 96, 96)])
def test_c3_full_mesh_path_for_path_on_windows(gpu, mesh, window):
    """The full mesh at 1024x1024, depth 12, n=2: the wavefront (and the
    megakernel) with quad-light NEE against the oracle's restatement of the
    production estimator on a window across the lit top of the mesh and one
    on the left wall and the floor."""
    w, sid, orc = mesh
    x, y, ww, wh = window
    st = dataclasses.replace(w.settings, samples=2)
    ref, _, _ = orc.render_split(st, window=window)
    for engine in (A.ENGINE_WAVEFRONT, A.ENGINE_MEGAKERNEL):
        img = gpu.render(sid, dataclasses.replace(st, engine=engine))
        near_exact(img[y:y + wh, x:x + ww], ref)


def test_c3_full_mesh_three_sigma_against_bsdf_only_reference(gpu, mesh):
    """The configured n=8 (64 spp), depth 12: the production estimator with
    quad-light NEE against the expectation of the reference's own estimator,
    which reaches the small emitter by BSDF sampling only (heavy-tailed
    per-pixel means, so 4x4-pixel blocks), on a 64x64 window across the lit
    top of the mesh."""
    w, sid, orc = mesh
    window = (448, 330, 64, 64)
    x, y, ww, wh = window
    st = w.settings
    mu_o, m2_o, _ = orc.render(st, want_m2=True, window=window)
    m2_g = np.zeros((st.height, st.width, 3), np.float32)
    mu_g = gpu.render(sid, st, m2=m2_g)
    mu_g, m2_g = mu_g[y:y + wh, x:x + ww], m2_g[y:y + wh, x:x + ww]
    va, vb = np.maximum(m2_g - mu_g ** 2, 0), np.maximum(m2_o - mu_o ** 2, 0)
    assert vb.mean() > va.mean()           # NEE lowers the variance
    z, diff, se = block_z(mu_g, m2_g, mu_o, m2_o, 64, 4)
    frac = (np.abs(z) > 3).mean()
    print(f"C3 window: {frac:.4f} of block channels beyond 3 sigma; mean {mu_g.mean():.5f} "
          f"(BSDF-only reference {mu_o.mean():.5f})")
    assert frac <= 0.03
    assert abs(diff.sum()) <= 3 * np.sqrt((se ** 2).sum())


def test_c4_batch_of_32_scenes_at_configured_sizes(gpu):
    jobs = W.sphere_batch(n_scenes=32, seed=4)
    sids = [gpu.upload(j.scene) for j in jobs]
    sts = [j.settings for j in jobs]
    paths = sum(st.width * st.height * st.samples ** 2 for st in sts)
    assert paths > 2e7 and len({(st.width, st.samples) for st in sts}) > 4
    singles = [gpu.render(s, st) for s, st in zip(sids, sts)]
    for key, block in ((0, 128), (3, 256), (2, 64)):
        for st in sts:
            st.sort_key, st.block_size = key, block
        batch = gpu.render_batch(sids, sts)
        for k, (a, b) in enumerate(zip(singles, batch)):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (key, block, k)
    for s in sids:
        gpu.free(s)


@pytest.mark.parametrize("name", ["three_spheres", "shapes", "cornell_box"])
def test_reference_golden_pngs_through_the_gpu(gpu, name):
    """Pencil's golden PNGs (tests/three_spheres.png, shapes.png,
    cornell_box.png of the reference) come from its default Whitted mode:
    the GPU megakernel in exact mode renders them at their golden size, the
    device tone map (pgpu_tonemap, ACES + gamma 2.2) makes the bytes, which
    are compared with the oracle's bytes (SHA-256-equal to the reference's
    three_spheres and shapes PNGs, within 1 LSB of cornell_box). Budget: the
    last bits of libm's cos/sin/pow on the device against the host's can move
    a soft-shadow sample or a byte at a rounding boundary, so at most 0.2% of
    bytes may differ, by at most 2 LSB for 99.9% of bytes."""
    scene, fx = load_golden(name)
    g = png_goldens()[name]
    r = g["render"]
    st = RenderSettings(width=r["width"], height=r["height"], samples=r["samples"],
                        max_depth=r["depth"], pathtrace=False, engine=A.ENGINE_MEGAKERNEL,
                        rng=A.RNG_PIXEL_SEQUENTIAL, glass=A.GLASS_BOTH_BRANCHES,
                        binary_tree=True)
    sid = gpu.upload(scene, fx["nodes"])
    hdr = gpu.render(sid, st)
    px = gpu.tonemap(hdr, A.TONEMAP_ACES)
    gpu.free(sid)
    ref_hdr, _, _ = O.Oracle(scene, fx["nodes"], fx["prims"]).render(st)
    ref = O.rgb8(ref_hdr, tonemap=1)
    assert list(px.shape) == g["shape"]
    d = np.abs(px.astype(int) - ref.astype(int))
    exact = hashlib.sha256(np.ascontiguousarray(px).tobytes()).hexdigest() == g.get("sha256")
    print(f"{name}: {(d > 0).mean():.6f} of bytes differ, max {d.max()} LSB; "
          f"SHA-256 equal to the reference PNG: {exact}")
    assert (d > 0).mean() <= 0.002
    assert (d > 2).mean() <= 0.001
