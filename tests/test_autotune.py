"""The autotuner's search on the host (pencil_b200/autotune.py), with the
device timing replaced by a synthetic cost: which candidates it tries, that
it keeps the best of each coordinate, that capacities stop at what half the
free memory holds, that the choice is applied to every settings object, and
that a second call with the same workload shape reads the cache."""
from __future__ import annotations

import json

import pytest

from pencil_b200 import _abi as A
from pencil_b200 import autotune as T
from pencil_b200.renderer import RenderSettings

torch = pytest.importorskip("torch")


class FakeScene:
    n_unified = 1000
    n_materials = 3
    lights = [object()]


class FakeCtx:
    """Stands in for GpuContext: renders do nothing, the cost is synthetic."""

    def __init__(self):
        self.calls = 0

    def render_device(self, sid, st, ptr):
        self.calls += 1

    def render_batch(self, sids, settings, device_ptrs):
        self.calls += 1


BEST = {"queue_capacity": 1 << 22, "refill_below": 16, "sort_key": 3, "block_size": 64}


def cost(st: RenderSettings) -> float:
    """A bowl whose minimum is BEST, separable by coordinate."""
    c = abs(st.queue_capacity.bit_length() - BEST["queue_capacity"].bit_length()) * 3.0
    c += abs(st.refill_below - BEST["refill_below"]) * 0.5
    c += 0.0 if st.sort_key == BEST["sort_key"] else 2.0 + st.sort_key * 0.1
    c += 0.0 if st.block_size == BEST["block_size"] else 1.0
    return 10.0 + c


@pytest.fixture
def tuner(monkeypatch, tmp_path):
    ctx = FakeCtx()
    settings = [RenderSettings(width=512, height=512, samples=8, pathtrace=True,
                               pathtrace_bounces=8)]
    monkeypatch.setattr(T, "CACHE", tmp_path / "autotune.json")
    monkeypatch.setattr(T, "_time_device", lambda c, render, reps: (render(), cost(settings[0]))[1])
    monkeypatch.setattr(torch, "empty", lambda *a, **k: torch.zeros(1))
    # 4 GiB free: half holds 2^22 paths at 512 bytes each, not 2^23
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda *a: (4 << 30, 8 << 30))
    return ctx, settings


def test_coordinate_search_finds_the_bowl_minimum(tuner):
    ctx, settings = tuner
    out = T.autotune(ctx, [0], settings, scene=FakeScene(), reps=1)
    for k, v in BEST.items():
        assert out[k] == v
        assert getattr(settings[0], k) == v          # applied to the settings
    assert settings[0].engine == A.ENGINE_WAVEFRONT
    assert out["cached"] is False
    assert out["ms"] == pytest.approx(10.0)
    tried = {t["queue_capacity"] for t in out["trials"]}
    # 2^24 paths in the frame, but half of the 4 GiB free holds 2^22 paths
    # at 512 bytes each: no capacity beyond that is tried
    assert tried == {1 << 20, 1 << 21, 1 << 22}
    assert len(out["trials"]) == 3 + len(T.REFILLS) + len(T.SORT_KEYS) + len(T.BLOCKS)
    assert ctx.calls == len(out["trials"])


def test_capacities_up_to_the_whole_frame(tuner, monkeypatch):
    ctx, settings = tuner
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda *a: (64 << 30, 80 << 30))
    out = T.autotune(ctx, [0], settings, scene=FakeScene(), reps=1, use_cache=False)
    tried = sorted({t["queue_capacity"] for t in out["trials"]})
    # room for 2^26 paths: every power of two below the frame's 2^24 paths,
    # then the whole frame as one chunk
    assert tried == [1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24]
    assert out["queue_capacity"] == BEST["queue_capacity"]
    # a frame smaller than every candidate is tried whole
    settings[0].width, settings[0].height, settings[0].samples = 64, 32, 4
    out = T.autotune(ctx, [0], settings, scene=FakeScene(), reps=1, use_cache=False)
    assert {t["queue_capacity"] for t in out["trials"]} == {64 * 32 * 16}


def test_second_call_reads_the_cache(tuner):
    ctx, settings = tuner
    first = T.autotune(ctx, [0], settings, scene=FakeScene(), reps=1)
    calls = ctx.calls
    cached = json.loads(T.CACHE.read_text())
    assert list(cached.values())[0]["sort_key"] == BEST["sort_key"]
    fresh = [RenderSettings(width=512, height=512, samples=8, pathtrace=True,
                            pathtrace_bounces=8)]
    again = T.autotune(ctx, [0], fresh, scene=FakeScene(), reps=1)
    assert again["cached"] is True and ctx.calls == calls    # no renders
    for k in BEST:
        assert again[k] == first[k] == getattr(fresh[0], k)
    # another shape is searched again
    other = [RenderSettings(width=256, height=256, samples=8, pathtrace=True,
                            pathtrace_bounces=8)]
    assert T.autotune(ctx, [0], other, scene=FakeScene(), reps=1)["cached"] is False


def test_signature_follows_the_workload_shape():
    a = [RenderSettings(width=64, height=64, samples=2, pathtrace=True, pathtrace_bounces=4)]
    b = [RenderSettings(width=64, height=64, samples=2, pathtrace=True, pathtrace_bounces=5)]
    s = FakeScene()
    assert T.signature(s, a) == T.signature(s, a)
    assert T.signature(s, a) != T.signature(s, b)
    t = FakeScene()
    t.n_unified = 1001
    assert T.signature(s, a) != T.signature(t, a)
