"""Pencil's HDR -> 8-bit output path (write_image, src/image_io.hpp:63-113;
tone curves, src/tonemap.hpp:27-61) on the device: pgpu_tonemap.

The device reproduces the host's gamma byte through 255 thresholds taken
with the host's own powf; that is exact when the host's gamma byte never
decreases, which the CPU test checks over every float in [0, 1]. The GPU
test compares bytes with the oracle's restatement (itself pinned to the
reference's golden PNGs) at the thresholds, one ulp below them, on random
values and on rendered images.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from pencil_b200 import _abi as A


def test_host_gamma_byte_is_monotone_over_all_floats():
    assert O.gamma_monotone() == 0


def gamma_thresholds() -> np.ndarray:
    """Smallest float32 in [0, 1] whose gamma byte (no tone curve) is >= k,
    k = 1..255, by bisection over bit patterns (all k at once)."""
    lo = np.zeros(255, np.uint32)
    hi = np.full(255, 0x3F800000, np.uint32)
    k = np.arange(1, 256)
    while np.any(lo < hi):
        mid = lo + (hi - lo) // 2
        v = mid.view(np.float32)
        byte = O.rgb8(np.repeat(v[:, None], 3, 1), tonemap=A.TONEMAP_NONE)[:, 0]
        up = byte >= k
        hi = np.where(up & (lo < hi), mid, hi)
        lo = np.where(~up & (lo < hi), mid + 1, lo)
    return lo.view(np.float32)


@pytest.mark.gpu
def test_device_tonemap_equals_host_bytes(gpu):
    t = gamma_thresholds()
    below = np.nextafter(t, np.float32(-np.inf)).astype(np.float32)
    rng = np.random.default_rng(12)
    vals = np.concatenate([t, below, rng.uniform(-0.5, 1.5, 60000).astype(np.float32),
                           np.exp(rng.normal(0, 3, 60000)).astype(np.float32),
                           np.array([0, -0.0, 1, 1e30, -1e30, np.inf, -np.inf], np.float32)])
    vals = vals[: len(vals) // 3 * 3].reshape(-1, 3)
    for mode in (A.TONEMAP_NONE, A.TONEMAP_ACES, A.TONEMAP_REINHARD):
        for exposure in (0.0, 1.5, -2.0):
            want = O.rgb8(vals, tonemap=mode, exposure=exposure)
            got = gpu.tonemap(vals, mode, exposure)
            assert np.array_equal(got, want), (mode, exposure, int((got != want).sum()))


@pytest.mark.gpu
def test_device_tonemap_of_renders(gpu):
    from conftest import load_golden
    for name in ("three_spheres", "shapes", "cornell_box"):
        _, fx = load_golden(name)
        hdr = fx["hdr_wh"]
        assert np.array_equal(gpu.tonemap(hdr), O.rgb8(hdr, tonemap=A.TONEMAP_ACES))


@pytest.mark.gpu
def test_device_tonemap_rejects_bad_arguments(gpu):
    with pytest.raises(A.GpuError) as e:
        gpu.tonemap(np.zeros((2, 2, 3), np.float32), tonemap=3)
    assert e.value.code == A.ERR_UNSUPPORTED
    assert gpu.tonemap(np.zeros((0, 3), np.float32)).shape == (0, 3)
