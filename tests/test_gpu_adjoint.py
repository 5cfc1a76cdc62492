"""The path-replay adjoint (pgpu_adjoint) through the C-ABI.

Checked against the FP64 CPU adjoint of the oracle (the same paths replayed,
gradients summed in double), against central finite differences with common
random numbers (h = 1e-3, same seeds), and by inverse rendering: a
torch.autograd.Function wraps render + adjoint (here, in the test harness
only) and Adam recovers hidden per-sphere albedos of the box scene.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from pencil_b200 import _abi as A
from pencil_b200 import workloads as W
from pencil_b200.renderer import RenderSettings

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel_err(a, b, floor):
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


@pytest.mark.parametrize("case", ["box", "prims"])
def test_adjoint_matches_fp64_cpu_adjoint(gpu, case):
    if case == "box":
        w, _, _ = W.adjoint_box(60, 32, 32, 2, 4, seed=9)
        scene, st = w.scene, w.settings
    else:
        from conftest import load_golden
        scene, fx = load_golden("prims_mix")
        st = RenderSettings(width=48, height=36, samples=2, pathtrace=True, pathtrace_bounces=6)
    sid = gpu.upload(scene)
    fwd = gpu.render(sid, st)
    dl = np.random.default_rng(1).normal(size=fwd.shape).astype(np.float32)
    nm, nl = scene.n_materials, len(scene.lights)
    da, de, dli, img = gpu.adjoint(sid, st, dl, nm, nl, want_image=True)
    # the replay renders the same samples as the forward render
    assert (rel_err(img, fwd, 1e-3) > 1e-4).mean() <= 0.005
    ca, ce, cl, _ = O.Oracle(scene).adjoint(st, dl)
    for g, c in ((da, ca), (de, ce), (dli, cl)):
        scale = max(np.abs(c).max(), 1e-12)
        # FP32 per-path sums on the GPU against FP64 on the CPU; paths whose
        # last-bit libm differences flip a decision are rare
        assert np.abs(g - c).max() <= 2e-3 * scale
    gpu.free(sid)


@pytest.mark.parametrize("res", [128, 512])
def test_adjoint_matches_central_differences(gpu, res):
    """Central differences with common random numbers (h = 1e-3, the same
    seeds on both sides) on the box with 1,000 spheres, 16 spp, depth 6; at
    512x512 this is the adjoint configuration itself."""
    w, target, first = W.adjoint_box(1000, res, res, 4, 6, seed=5)
    scene, st = w.scene, w.settings
    sid = gpu.upload(scene)
    fwd = gpu.render(sid, st)
    dl = (2.0 * (fwd - 0.5 * fwd.mean())).astype(np.float32)    # an L2-style weight
    nm, nl = scene.n_materials, len(scene.lights)
    da, de, dli, _ = gpu.adjoint(sid, st, dl, nm, nl)
    mats = scene.material_array().copy()
    big = np.argsort(-np.abs(da[first:]).sum(axis=1))[:6] + first
    h = 1e-3
    for m in big:
        for c in range(3):
            if abs(da[m, c]) < 1e-3 * np.abs(da).max():
                continue
            mp, mm = mats.copy(), mats.copy()
            mp["albedo"][m, c] += h
            mm["albedo"][m, c] -= h
            gpu.update_materials(sid, mp)
            lp = float((dl.astype(np.float64) * gpu.render(sid, st)).sum())
            gpu.update_materials(sid, mm)
            lm = float((dl.astype(np.float64) * gpu.render(sid, st)).sum())
            fd = (lp - lm) / (2 * h)
            assert abs(da[m, c] - fd) <= 0.02 * abs(fd) + 1e-6 * np.abs(da).max(), (m, c, da[m, c], fd)
    gpu.update_materials(sid, mats)
    gpu.free(sid)


class RenderAlbedo(torch.autograd.Function):
    """image = render(albedos of materials [first, first + n)); the backward
    pass is pgpu_adjoint. The adjoint replays a different set of samples than
    the forward image (seed decorrelated): with shared samples the gradient
    of an L2 loss, 2 (I - target) dI/da, would correlate the noise of I with
    that of dI/da and be biased."""

    @staticmethod
    def forward(ctx, albedo, gpu, sid, st, mats, first):
        m = mats.copy()
        m["albedo"][first:first + len(albedo)] = albedo.detach().cpu().numpy()
        gpu.update_materials(sid, m)
        img = gpu.render(sid, st)
        ctx.gpu, ctx.sid, ctx.st, ctx.first, ctx.n = gpu, sid, st, first, len(albedo)
        ctx.nm, ctx.nl = len(m), 0
        return torch.from_numpy(img)

    @staticmethod
    def backward(ctx, grad_img):
        import dataclasses
        dl = grad_img.detach().cpu().numpy().astype(np.float32)
        st = dataclasses.replace(ctx.st, seed=(ctx.st.seed * 2654435761 + 97) & 0xFFFFFFFF)
        da, _, _, _ = ctx.gpu.adjoint(ctx.sid, st, dl, ctx.nm, 1)
        g = torch.from_numpy(da[ctx.first:ctx.first + ctx.n].astype(np.float32))
        return g, None, None, None, None, None


def inverse_render(gpu, n_spheres, res, samples, depth, steps, lr0, lr1, fresh_samples):
    """Adam on the per-sphere albedos from 0.5 towards the hidden target, the
    learning rate decaying exponentially from lr0 to lr1. Progress is
    measured with common random numbers (the target's seed), so the Monte
    Carlo noise of target and estimate cancel, and on the spheres visible in
    at least 20 pixel centres (hidden ones get no gradient)."""
    wt, target_alb, first = W.adjoint_box(n_spheres, res, res, samples, depth, seed=5)
    sid = gpu.upload(wt.scene)
    st = wt.settings
    target = torch.from_numpy(gpu.render(sid, st))
    mats = wt.scene.material_array().copy()
    ys, xs = np.mgrid[0:res, 0:res]
    uv = np.stack([(xs + 0.5) / res, 1 - (ys + 0.5) / res], -1).reshape(-1, 2).astype(np.float32)
    prim, _ = gpu.primary_hits(sid, uv)
    n_box = wt.scene.n_prims - n_spheres
    visible = np.bincount(prim[prim >= n_box] - n_box, minlength=n_spheres) >= 20

    def crn_loss(a):
        st.seed = 0
        with torch.no_grad():
            img = RenderAlbedo.apply(a, gpu, sid, st, mats, first)
        return float(((img - target) ** 2).sum())

    alb = torch.full((n_spheres, 3), 0.5, requires_grad=True)
    loss0 = crn_loss(alb)
    opt = torch.optim.Adam([alb], lr=lr0)
    sched = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=(lr1 / lr0) ** (1.0 / steps))
    for k in range(steps):
        st.seed = k + 1 if fresh_samples else 0
        opt.zero_grad()
        img = RenderAlbedo.apply(alb, gpu, sid, st, mats, first)
        loss = ((img - target) ** 2).sum()
        loss.backward()
        opt.step()
        sched.step()
        with torch.no_grad():
            alb.clamp_(0.0, 1.0)
    loss1 = crn_loss(alb)
    err0 = np.abs(0.5 - target_alb)[visible].mean()
    err = np.abs(alb.detach().numpy() - target_alb)[visible].mean()
    gpu.free(sid)
    return loss0, loss1, err0, err, int(visible.sum())


def test_inverse_rendering_small(gpu):
    loss0, loss1, err0, err, nv = inverse_render(gpu, 60, 64, 2, 4, 60, 0.05, 0.05,
                                                 fresh_samples=False)
    print(f"inverse rendering (small): CRN loss {loss0:.2f} -> {loss1:.2f}, "
          f"mean |albedo error| of {nv} visible spheres {err0:.4f} -> {err:.4f}")
    assert loss1 < 0.05 * loss0
    assert err < 0.3 * err0


def test_inverse_rendering_box_200_adam_steps(gpu):
    """The adjoint configuration: 1,000 spheres, 512x512, 16 spp, depth 6,
    fresh samples at every step, 200 Adam steps."""
    loss0, loss1, err0, err, nv = inverse_render(gpu, 1000, 512, 4, 6, 200, 0.02, 0.002,
                                                 fresh_samples=True)
    print(f"inverse rendering: CRN loss {loss0:.1f} -> {loss1:.1f}, "
          f"mean |albedo error| of {nv} visible spheres {err0:.4f} -> {err:.4f}")
    assert loss1 < 0.25 * loss0
    assert err < 0.5 * err0
