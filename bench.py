#!/usr/bin/env python
"""Benchmark of the GPU path-tracing core.

Workload (the sphere-cloud configuration): 100,000 seeded random spheres
(60/30/10 diffuse/metal/glass), one directional light, sky 0.3; 1280x720,
n=4 (16 spp), depth 8; 14,745,600 paths per frame. A step renders one frame.

  value   Mpaths/s of the wavefront engine with the scene resident in HBM and
          the image written to device memory (CUDA events on the render
          stream, L2 flushed between steps outside the timed events)
  e2e     the same metric through the C-ABI as Pencil's --gpu mode calls it:
          every step uploads the scene from pinned host memory
          (pgpu_upload_scene), renders into a pinned host image (pgpu_render)
          and frees the scene
  extras  the megakernel's Mpaths/s on the same frame (the images are
          bit-identical, so equal RMSE), Mrays/s, per-kernel roofline

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank renders the frame with its own sample
offset (weak scaling: per-GPU work fixed) and the HDR images are summed with
one NCCL all-reduce per step, inside the timed region. `--impl reference`
times the reference CPU renderer (oracle/_ref, built from the reference's
own sources; the C oracle port where it is absent) on a bounded sample of
the same workload on this host's cores.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = ("Mpaths/s & Mrays/s at equal RMSE, wavefront vs megakernel (1 B200); "
          "adjoint ms/grad")
WORKLOAD = "sphere_cloud_100k_1280x720_n4_16spp_depth8"
# The bounded CPU sample: the full frame at n=2 (4 spp instead of 16; the
# per-path work is the same), 240 of Pencil's 64x64 tiles, so every host
# thread gets many tiles and none idles at the end.
CPU_SAMPLE = (1280, 720, 2, 8)     # width, height, n, depth
CPU_RUNS = 3                       # timed runs (median) after one warm-up run
# Window of the frame whose paths the oracle replays to count the
# reference-order traversal work (algorithmic bytes).
COUNT_WINDOW = (480, 270, 320, 180)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the adjoint, batch and image-quality measurements")
    ap.add_argument("--profile-pencil-tree", action="store_true",
                    help="mesh profile case: the wide traversals on Pencil's tree")
    ap.add_argument("--profile-case", choices=["wavefront", "megakernel", "mesh",
                                               "mesh_megakernel", "adjoint", "lbvh", "tonemap"],
                    default=None,
                    help="render the workload once, kernels launched one by one (for ncu)")
    ap.add_argument("--profile-scale", type=int, default=1,
                    help="divide the image width and height by this (smaller ncu cases)")
    ap.add_argument("--arena-sizes", action="store_true",
                    help="traversal cost per node visit on mesh arenas of 15 MB to 1 GB "
                         "(one JSON line per size)")
    ap.add_argument("--profile-counts", action="store_true",
                    help="with --profile-case: also render once with ray counters and "
                         "print them (run without ncu)")
    return ap.parse_args()


# ---- clocks ---------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples (every 200 ms) while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.out.flush()
        rows = []
        for line in Path(self.out.name).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


# ---- CPU reference ----------------------------------------------------------------
def cpu_reference_run(scene, steps: int, warmup: int) -> dict:
    """Time the reference CPU renderer on the bounded sample: seconds per run."""
    from oracle import oracle as O
    w, h, n, depth = CPU_SAMPLE
    threads = os.cpu_count() or 1
    paths = w * h * n * n
    if O.ref_available():
        _, info = O.ref_render(scene, w, h, n, depth, True, threads=threads,
                               repeat=warmup + steps, want_image=False)
        secs = info["seconds"][warmup:]
        kind = "reference"
    else:
        from pencil_b200.renderer import RenderSettings
        orc = O.Oracle(scene)
        st = RenderSettings(width=w, height=h, samples=n, pathtrace=True, pathtrace_bounces=depth)
        secs = []
        for k in range(warmup + steps):
            t = time.perf_counter()
            orc.render(st, threads=threads)
            if k >= warmup:
                secs.append(time.perf_counter() - t)
        kind = "port"
    med = statistics.median(secs)
    return {"value": paths / med / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": kind,
            "sample": f"the same 100k-sphere frame at {w}x{h}, n={n} ({n*n} spp), depth {depth}: "
                      f"{paths} paths and {-(-w // 64) * -(-h // 64)} 64x64 tiles per run, "
                      f"median of {len(secs)} runs after {warmup} warm-up",
            "seconds": secs}


def cpu_batch_sample(jobs) -> dict:
    """The reference CPU renderer on a seeded subset of the batch's scenes
    (one run each, all host threads), as a per-path rate."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    if not O.ref_available():
        return {"value": None, "unit": "Mpaths/s", "cores": threads, "kind": "reference",
                "sample": "unavailable: the reference renderer is not built"}
    secs, paths = 0.0, 0
    for j in jobs:
        st = j.settings
        _, info = O.ref_render(j.scene, st.width, st.height, st.samples, st.pathtrace_bounces,
                               True, threads=threads, repeat=1, want_image=False)
        secs += float(info["seconds"][0])
        paths += st.width * st.height * st.samples ** 2
    return {"value": paths / secs / 1e6, "unit": "Mpaths/s", "cores": threads,
            "kind": "reference", "scenes": len(jobs), "paths": paths, "seconds": secs,
            "sample": f"every 32nd of the 256 scenes ({len(jobs)}), one run each, "
                      "extrapolated per path"}


def reference_order_counts(scene, settings) -> dict:
    """Algorithmic work per ray of the frame's paths, counted by the oracle
    on COUNT_WINDOW: its replay of the production estimator walks Pencil's
    binary tree in Pencil's own order (BVHNode::hit / occluded: left child,
    then right, every box tested), so the node and primitive counts are the
    reference algorithm's for the very rays the GPU traces."""
    import dataclasses

    from oracle import oracle as O
    t0 = time.perf_counter()
    _, _, cnt = O.Oracle(scene).render_split(dataclasses.replace(settings),
                                             window=COUNT_WINDOW)
    ext, sh = int(cnt[O.CNT_EXTENSION_RAYS]), int(cnt[O.CNT_SHADOW_RAYS])
    x, y, w, h = COUNT_WINDOW
    paths = w * h * settings.samples ** 2
    return {"window": list(COUNT_WINDOW), "paths": paths,
            "ext_rays_per_path": ext / paths, "shadow_rays_per_path": sh / paths,
            "ext_nodes_per_ray": float(cnt[O.CNT_EXT_NODES]) / max(ext, 1),
            "ext_prim_bytes_per_ray": float(cnt[O.CNT_EXT_PRIM_BYTES]) / max(ext, 1),
            "shadow_nodes_per_ray": float(cnt[O.CNT_SH_NODES]) / max(sh, 1),
            "shadow_prim_bytes_per_ray": float(cnt[O.CNT_SH_PRIM_BYTES]) / max(sh, 1),
            "seconds": time.perf_counter() - t0}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from pencil_b200 import workloads as W
    wl = W.sphere_cloud()
    steps, warmup = max(args.steps, 1), max(args.warmup, 0)
    # each step is one bounded-sample render; keep the whole run to a few minutes
    steps = min(steps, 8)
    warmup = min(warmup, 1)
    cb = cpu_reference_run(wl.scene, steps, warmup)
    ms = statistics.median(cb["seconds"]) * 1e3
    line = {"metric": METRIC, "value": cb["value"], "unit": "Mpaths/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": WORKLOAD, "sample": cb["sample"], "threads": cb["cores"]},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---- GPU ----------------------------------------------------------------------------
def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def ncu_per_ray() -> dict:
    """Per-extension-ray DRAM bytes, L2 sectors and L2 throughput of one
    wf_extend launch, from the committed ncu summary
    (profiles/wf_extend_sphere_cloud.txt), where present."""
    p = ROOT / "profiles" / "wf_extend_sphere_cloud.txt"
    out = {}
    if not p.exists():
        return out
    text = p.read_text()
    for key in ("dram_bytes_per_ray", "l2_sectors_per_ray", "l2_throughput_pct",
                "dram_throughput_pct", "l1_lsu_wavefronts_pct"):
        m = re.search(key + r":\s*([0-9.eE+-]+)", text)
        if m:
            out[key] = float(m.group(1))
    return out


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist
    from pencil_b200 import _abi as A
    from pencil_b200 import workloads as W
    from pencil_b200.renderer import GpuContext, RenderSettings, RenderStats

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from pencil_b200.distributed import combine, shard_settings
    wl = W.sphere_cloud()
    # every rank renders the whole frame with its own samples (weak scaling)
    st: RenderSettings = shard_settings(wl.settings, rank, world)
    paths_per_frame = st.width * st.height * st.samples ** 2
    ctx = GpuContext(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    sid = ctx.upload(wl.scene)
    img = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    # launch parameters of the wavefront engine, picked by the autotuner
    # (outside the timed region)
    from pencil_b200.autotune import autotune
    tuned = autotune(ctx, [sid], [st], scene=wl.scene, use_cache=False)
    tuned = {**{k: tuned[k] for k in ("queue_capacity", "refill_below", "sort_key", "block_size",
                                      "ms")},
             "trials": [[t["queue_capacity"], t["refill_below"], t["sort_key"], t["block_size"],
                         round(t["ms"], 3)] for t in tuned.get("trials", [])]}

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(engine: int, steps: int, warmup: int, clocks=None):
        st.engine = engine
        for _ in range(warmup):
            ctx.render_device(sid, st, img.data_ptr())
            with torch.cuda.stream(stream):
                combine(img, world)
        evs = []
        barrier()
        cm = clocks if clocks is not None else _Null()
        with cm:
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.render_device(sid, st, img.data_ptr())
                with torch.cuda.stream(stream):
                    combine(img, world)        # the frame's one exchange
                e1.record(stream)
                evs.append((e0, e1))
            barrier()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        t = torch.tensor([ms], device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()) / steps

    clocks = ClockSampler(local)
    ms_wf = timed(A.ENGINE_WAVEFRONT, args.steps, args.warmup, clocks)
    clk = clocks.summary()
    mk_steps = max(2, min(args.steps, 5))
    # the plain megakernel on the same 4-wide tree (the baseline), and on
    # Pencil's binary tree
    ms_mk = timed(A.ENGINE_MEGAKERNEL, mk_steps, 1)
    st.binary_tree = True
    ms_mk_bin = timed(A.ENGINE_MEGAKERNEL, mk_steps, 1)
    st.binary_tree = False
    value = paths_per_frame * world / (ms_wf * 1e-3) / 1e6
    mk_value = paths_per_frame * world / (ms_mk * 1e-3) / 1e6

    # instrumented runs (outside the timed region): ray/node counts, kernel times
    st.engine = A.ENGINE_WAVEFRONT
    cnt = RenderStats()
    st.count_rays, st.count_nodes = True, True
    ctx.render(sid, st, stats=cnt)
    st.count_rays, st.count_nodes = False, False
    prof = RenderStats()
    st.profile_kernels = True
    ctx.render(sid, st, stats=prof)
    ctx.render(sid, st, stats=prof)
    st.profile_kernels = False
    rays = cnt.extension_rays + cnt.shadow_rays
    mrays = rays * world / (ms_wf * 1e-3) / 1e6

    # roofline of the dominant kernel (closest-hit traversal, wf_extend):
    # algorithmic bytes of the reference algorithm per extension ray -- 32 B
    # per binary node Pencil's walk visits, the primitive records it tests,
    # and the queue traffic of one ray (origin + direction read, hit record
    # written, queue slot read: 52 B) -- counted by the oracle on rank 0
    kms = prof.kernel_ms
    dominant = max(("extend", "shade", "shadow", "generate", "accumulate"), key=lambda k: kms[k])
    chunk = st.queue_capacity if st.queue_capacity > 0 else paths_per_frame
    n_ext_launches = max(1, -(-paths_per_frame // max(1, chunk)) * st.pathtrace_bounces)
    ext_launch_ms = kms["extend"] / n_ext_launches
    rays_per_launch = cnt.extension_rays / n_ext_launches
    peaks = measured_peaks()
    ncu = ncu_per_ray()
    ref_counts = None
    if rank == 0:
        try:
            ref_counts = reference_order_counts(wl.scene, dataclasses.replace(st))
        except Exception as ex:  # noqa: BLE001
            ref_counts = {"error": str(ex)}
    roof = {"kernel": "wf_extend", "bound": "hbm", "unit": "GB/s", "peak": peaks["hbm_gbs"],
            "peak_source": peaks["source"], "launches": n_ext_launches,
            "avg_launch_ms": ext_launch_ms, "rays_per_launch": rays_per_launch,
            "dominant_kernel_by_time": dominant, "kernel_ms": kms,
            "gpu_wide_nodes_per_ray": cnt.ext_node_visits / max(1, cnt.extension_rays)}
    if ref_counts and "ext_nodes_per_ray" in ref_counts:
        per_ray = (32.0 * ref_counts["ext_nodes_per_ray"] + ref_counts["ext_prim_bytes_per_ray"]
                   + 52.0)
        alg = per_ray * rays_per_launch
        achieved = alg / (ext_launch_ms * 1e-3) / 1e9
        roof.update({"achieved": achieved, "frac": achieved / peaks["hbm_gbs"],
                     "algorithmic_bytes_per_launch": alg,
                     "algorithmic_bytes_per_ray": per_ray,
                     "reference_order": ref_counts})
    else:
        roof.update({"achieved": None, "frac": None, "reference_order": ref_counts})
    # what the memory system actually carried (ncu, one launch, scaled per ray)
    roof["traffic"] = (ncu["dram_bytes_per_ray"] * rays_per_launch
                       if "dram_bytes_per_ray" in ncu else None)
    if roof["traffic"] is not None:
        dram_gbs = roof["traffic"] / (ext_launch_ms * 1e-3) / 1e9
        roof["dram_achieved_gbs"] = dram_gbs
        roof["dram_frac"] = dram_gbs / peaks["hbm_gbs"]
    if "l2_sectors_per_ray" in ncu:
        l2_bytes = 32.0 * ncu["l2_sectors_per_ray"] * rays_per_launch
        roof["l2_bytes_per_launch"] = l2_bytes
        roof["l2_achieved_gbs"] = l2_bytes / (ext_launch_ms * 1e-3) / 1e9
    if "l2_throughput_pct" in ncu:
        roof["l2_frac"] = ncu["l2_throughput_pct"] / 100.0
    if "l1_lsu_wavefronts_pct" in ncu:
        roof["l1_data_pipe_frac"] = ncu["l1_lsu_wavefronts_pct"] / 100.0
    # the memory level the counters show busiest: "bound" keeps the class
    # (memory, no tensor work); this names the unit and its busy fraction
    levels = {k: roof[f] for k, f in (("dram", "dram_frac"), ("l2", "l2_frac"),
                                      ("l1_data_pipe", "l1_data_pipe_frac")) if f in roof}
    if levels:
        top = max(levels, key=levels.get)
        roof["bound_by_counters"] = {"unit": top, "frac": levels[top]}
    roof["limiter"] = ("the L1 data pipe serving scattered node loads (its lsu wavefronts at "
                       "l1_data_pipe_frac of peak in one ncu launch) and the latency of those "
                       "loads (long-scoreboard stalls); DRAM and L2 fractions well below 1, and "
                       "the time per node visit does not change between arenas of 15 MB and "
                       "977 MB; frac above 1 means the kernel finishes the reference "
                       "algorithm's node traffic faster than HBM could stream it")
    # the frame as a whole, per the same definition: bytes per path of every
    # segment (node/primitive bytes + ray, hit and path state read and
    # written, 192 B) and every shadow ray
    if ref_counts and "ext_nodes_per_ray" in ref_counts:
        per_path = (ref_counts["ext_rays_per_path"] *
                    (32.0 * ref_counts["ext_nodes_per_ray"] + ref_counts["ext_prim_bytes_per_ray"]
                     + 192.0) +
                    ref_counts["shadow_rays_per_path"] *
                    (32.0 * ref_counts["shadow_nodes_per_ray"] +
                     ref_counts["shadow_prim_bytes_per_ray"] + 48.0))
        roof["frame"] = {"bytes_per_path": per_path,
                         "achieved_gbs": per_path * value * 1e6 / 1e9 / world}

    # e2e through the C-ABI with host buffers
    e2e = None
    if not args.no_e2e:
        host_img = torch.empty((st.height, st.width, 3), dtype=torch.float32).pin_memory()
        out_np = host_img.numpy()
        h2d = ctx.scene_info(sid)["device_bytes"]   # the arena the upload copies
        d2h = out_np.nbytes
        ctx.render(sid, st, out=out_np)
        # Pencil builds its BVH when it parses the scene (ParsedScene::finalize);
        # its --gpu render hands that tree over, so it is built outside the loop
        nodes, _ = wl.scene.build_bvh()
        times, phases = [], []
        for k in range(args.warmup + args.steps):
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            s2 = ctx.upload(wl.scene, nodes)
            t1 = time.perf_counter()
            ctx.render(s2, st, out=out_np)
            t2 = time.perf_counter()
            ctx.free(s2)
            t3 = time.perf_counter()
            if k >= args.warmup:
                times.append(t3 - t0)
                phases.append((t1 - t0, t2 - t1, t3 - t2))
        sec = float(np.mean(times))
        t = torch.tensor([sec], device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec = float(t.item())
        ph = np.mean(np.array(phases), axis=0) * 1e3
        e2e = {"value": paths_per_frame * world / sec / 1e6, "unit": "Mpaths/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": sec * 1e3,
               "ms_upload_render_free": [round(float(x), 3) for x in ph]}

    extras = {}
    if rank == 0 and not args.no_extras:
        extras = measure_extras(ctx, sid, st, img, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_reference_run(wl.scene, CPU_RUNS, 1)
            cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "Mpaths/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {ex}"}

    launches_per_frame = prof.kernel_launches
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_wf,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded numpy scene; no dataset)",
            "config": {"workload": WORKLOAD, "engine": "wavefront", "spheres": 100000,
                       "width": st.width, "height": st.height, "spp": st.samples ** 2,
                       "depth": st.pathtrace_bounces, "paths_per_step": paths_per_frame * world,
                       "l2": "256 MiB memset between steps, outside the timed events",
                       "autotuned": tuned,
                       "parallelism": f"weak: {world} GPU(s), distinct sample offsets, "
                                      "NCCL all-reduce of the image per step" if world > 1
                                      else "1 GPU"},
            "mrays_per_s": mrays,
            "rays_per_step": rays,
            # Pencil's own count (RenderStats::rays_traced: one per trace /
            # trace_path call), for comparison with the reference's figures
            "reference_rays_per_step": cnt.rays_traced * world,
            "reference_mrays_per_s": cnt.rays_traced * world / (ms_wf * 1e-3) / 1e6,
            "megakernel": {"value": mk_value, "unit": "Mpaths/s", "ms_per_step": ms_mk,
                           "tree": "4-wide (the tree the wavefront walks)"},
            "megakernel_binary_tree": {"value": paths_per_frame * world / (ms_mk_bin * 1e-3) / 1e6,
                                       "unit": "Mpaths/s", "ms_per_step": ms_mk_bin,
                                       "tree": "Pencil's binary tree"},
            "wavefront_over_megakernel": ms_mk / ms_wf,
            "equal_rmse": "bit-identical images (same estimator, same random numbers)",
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
            "gpu_launches": launches_per_frame * args.steps,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    ctx.free(sid)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def _event_ms(stream, fn, reps: int) -> float:
    """Mean ms of fn() over `reps` calls after two untimed ones (a repeated
    frame shape runs as a CUDA graph from its second call on)."""
    import torch
    fn()
    fn()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def measure_extras(ctx, sid, st, img, stream) -> dict:
    """Outside the timed region: image quality against a 4096-spp render of
    the bench frame, the adjoint of the box configuration, the batch of 256
    uneven scenes and the triangle-mesh configuration."""
    import dataclasses

    import torch
    from pencil_b200 import _abi as A
    from pencil_b200 import workloads as W
    out = {"quality": measure_quality(ctx, sid, st, stream)}
    # adjoint of the box configuration: 1,000 spheres, 512x512, 16 spp, depth 6
    wa, _, _ = W.adjoint_box()
    sa = ctx.upload(wa.scene)
    ast = wa.settings
    buf = torch.empty((ast.height, ast.width, 3), dtype=torch.float32, device="cuda")
    fwd_ms = _event_ms(stream, lambda: ctx.render_device(sa, ast, buf.data_ptr()), 5)
    dl = np.random.default_rng(0).normal(size=(ast.height, ast.width, 3)).astype(np.float32)
    from pencil_b200.renderer import RenderStats
    adj = []
    for _ in range(4):
        s_ = RenderStats()
        ctx.adjoint(sa, ast, dl, wa.scene.n_materials, len(wa.scene.lights), stats=s_)
        adj.append(s_.device_ms)
    adj_ms = float(np.median(adj[1:]))
    out["adjoint"] = {"workload": "adjoint_box_1000spheres_512x512_16spp_depth6",
                      "ms_per_grad": adj_ms, "forward_ms": fwd_ms,
                      "grad_over_forward": adj_ms / fwd_ms,
                      "parameters": 3 * wa.scene.n_materials + 3 * len(wa.scene.lights)}
    ctx.free(sa)
    # batch: 256 uneven scenes in one launch sequence against one at a time
    jobs = W.sphere_batch()
    sids = [ctx.upload(j.scene) for j in jobs]
    sts = [j.settings for j in jobs]
    outs = [torch.empty((x.height, x.width, 3), dtype=torch.float32, device="cuda") for x in sts]
    ptrs = [o.data_ptr() for o in outs]
    paths = sum(x.width * x.height * x.samples ** 2 for x in sts)
    for x in sts:
        x.queue_capacity, x.refill_below, x.sort_key, x.block_size = 1 << 24, 16, 0, 0
    fixed_ms = _event_ms(stream, lambda: ctx.render_batch(sids, sts, device_ptrs=ptrs), 2)
    # the batch's launch parameters from the autotuner (capacity, refill,
    # sort key, block size), timed once each
    from pencil_b200.autotune import autotune
    tuned = autotune(ctx, sids, sts, reps=1, use_cache=False)
    batch_ms = _event_ms(stream, lambda: ctx.render_batch(sids, sts, device_ptrs=ptrs), 2)

    def one_by_one(engine):
        for sid_, x, p_ in zip(sids, sts, ptrs):
            x.engine = engine
            ctx.render_device(sid_, x, p_)
    seq_ms = _event_ms(stream, lambda: one_by_one(A.ENGINE_WAVEFRONT), 1)
    mk_ms = _event_ms(stream, lambda: one_by_one(A.ENGINE_MEGAKERNEL), 1)
    for x in sts:
        x.engine = A.ENGINE_WAVEFRONT
    out["batch"] = {"workload": "256 random-sphere scenes, 10-50,000 spheres, 128/256/512 "
                                "squared, 1/4/16/64 spp, depth 8",
                    "paths": paths, "batched_mpaths_s": paths / batch_ms / 1e3,
                    "batched_fixed_mpaths_s": paths / fixed_ms / 1e3,
                    "fixed_params": {"queue_capacity": 1 << 24, "refill_below": 16,
                                     "sort_key": 0, "block_size": 128},
                    "autotuned": {k: tuned[k] for k in ("queue_capacity", "refill_below",
                                                         "sort_key", "block_size")},
                    "one_by_one_wavefront_mpaths_s": paths / seq_ms / 1e3,
                    "one_by_one_megakernel_mpaths_s": paths / mk_ms / 1e3,
                    "batched_ms": batch_ms, "batched_fixed_ms": fixed_ms,
                    "one_by_one_wavefront_ms": seq_ms,
                    "one_by_one_megakernel_ms": mk_ms}
    for s_ in sids:
        ctx.free(s_)
    try:
        out["batch"]["cpu_baseline"] = cpu_batch_sample(jobs[::32])
    except Exception as ex:  # noqa: BLE001
        out["batch"]["cpu_baseline"] = {"value": None, "sample": f"failed: {ex}"}
    out["mesh"] = measure_mesh(ctx, stream)
    out["bvh_build"] = measure_bvh_build(ctx, stream)
    return out


def _reference_image(ctx, sid, st, window, frames: int = 64, n: int = 8):
    """Mean of `frames` renders of n x n spp with distinct sample offsets,
    and the relative RMSE of that mean's own noise (from its two halves)."""
    from pencil_b200.renderer import RenderStats
    halves = [np.zeros((window[3], window[2], 3)), np.zeros((window[3], window[2], 3))]
    q = dataclasses.replace(st, samples=n)
    ms = 0.0
    for k in range(frames):
        q.sample_offset = (k + 1000) * n * n
        s_ = RenderStats()
        halves[k * 2 // frames] += ctx.render_window(sid, q, window, stats=s_)
        ms += s_.device_ms
    a, b = halves[0] / (frames // 2), halves[1] / (frames // 2)
    ref = 0.5 * (a + b)
    noise = float(np.sqrt(((a - b) ** 2).mean()) / 2 / ref.mean())
    return ref, noise, ms


def _equal_rmse_point(ctx, sid, st, window, ref, noise, target=0.01, max_spp=4096,
                      ref_spp=4096) -> dict:
    """The samples per pixel at which the production estimator's image is
    within `target` relative RMSE of `ref`, and the device time of both
    engines to render the window at that point. Model: e^2 = a / spp +
    noise^2 (noise: the reference's own), a from a 16-spp render; the point
    is raised until the measured e meets the target (spp <= max_spp). Up to
    64 x 64 spp one render; beyond, the mean of several 64 x 64 renders with
    distinct sample offsets (the same estimator: independent samples)."""
    from pencil_b200 import _abi as A
    from pencil_b200.renderer import RenderStats

    def rmse(img):
        return float(np.sqrt(((img - ref) ** 2).mean()) / ref.mean())

    def truth(e):
        # RMSE against the converged image: the reference's own noise removed
        return float(np.sqrt(max(e * e - noise * noise, 0.0)))

    def plan(spp):
        if spp <= 4096:
            n = max(1, int(np.ceil(np.sqrt(spp))))
            return n, 1
        return 64, int(np.ceil(spp / 4096))

    q = dataclasses.replace(st, engine=A.ENGINE_WAVEFRONT, samples=4)
    e16 = rmse(ctx.render_window(sid, q, window))
    a = 16.0 * truth(e16) ** 2
    out = {"rel_rmse_16spp": e16, "reference_noise_rel_rmse": noise,
           "criterion": f"relative RMSE against the converged image (the {ref_spp}-spp "
                        "reference with its own measured noise removed) <= 1%"}
    n, reps = plan(min(max_spp, a / target ** 2))
    res = {}
    for _ in range(8):
        res = {}
        for name, eng in (("wavefront", A.ENGINE_WAVEFRONT), ("megakernel", A.ENGINE_MEGAKERNEL)):
            q = dataclasses.replace(st, engine=eng, samples=n)
            img = np.zeros((window[3], window[2], 3))
            ms = 0.0
            for r in range(reps):
                q.sample_offset = r * n * n
                s_ = RenderStats()
                img += ctx.render_window(sid, q, window, stats=s_)
                ms += s_.device_ms
            img /= reps
            paths = window[2] * window[3] * n * n * reps
            e = rmse(img)
            res[name] = {"ms": ms, "mpaths_s": paths / ms / 1e3,
                         "rel_rmse_vs_reference": e, "rel_rmse_vs_converged": truth(e)}
        spp = n * n * reps
        if res["wavefront"]["rel_rmse_vs_converged"] <= target or spp >= max_spp:
            break
        n, reps = plan(min(max_spp, spp * 1.15))
        if n * n * reps <= spp:
            n, reps = (n + 1, 1) if reps == 1 and n < 64 else (64, reps + 1)
    out.update({"reachable": res["wavefront"]["rel_rmse_vs_converged"] <= target,
                "spp": n * n * reps, "n": n, "renders": reps, **res,
                "wavefront_over_megakernel": res["megakernel"]["ms"] / res["wavefront"]["ms"]})
    return out


def measure_quality(ctx, sid, st, stream) -> dict:
    """Image quality at the north star's operating point (relative RMSE <=
    1% against a 4096-spp reference).

    Sphere cloud, the 640x360 middle of the full 1280x720 frame (the dense
    part of the cloud), rendered as windows of the frame: the reference
    image is the reference's own estimator -- trace_path with both
    dielectric branches (the megakernel's exact glass mode) -- at 4096 spp,
    as 64 renders of 64 spp with distinct sample offsets. Mesh box (the
    displaced icosphere, quad light) at 256x256, the wavefront with the
    launch parameters the autotuner picks for that frame: reference 32768 spp of the
    production estimator (32 renders of 1024 spp; at 4096 spp its own noise,
    1.3%, would hide the 1% criterion), the point searched up to 16384 spp; the reference's own estimator (BSDF sampling only: the small emitter
    is found by chance) at 4096 spp is measured against it too."""
    from pencil_b200 import _abi as A
    from pencil_b200 import workloads as W
    out = {}
    window = (320, 180, 640, 360)
    t0 = time.perf_counter()
    qref = dataclasses.replace(st, engine=A.ENGINE_MEGAKERNEL, glass=A.GLASS_BOTH_BRANCHES)
    ref, noise, ref_ms = _reference_image(ctx, sid, qref, window)
    out["sphere_cloud"] = {"window": list(window),
                           "reference": "trace_path with both glass branches, 4096 spp",
                           "reference_seconds": time.perf_counter() - t0,
                           **_equal_rmse_point(ctx, sid, st, window, ref, noise)}
    # mesh box at 256x256
    wm = W.mesh_box(width=256, height=256)
    nodes, _ = wm.scene.build_bvh()
    ctx.set_traversal_tree(A.TRAVERSAL_LBVH)      # the mesh's configuration (measure_mesh)
    try:
        sm = ctx.upload(wm.scene, nodes)
    finally:
        ctx.set_traversal_tree(A.TRAVERSAL_UPLOADED)
    sm_st = dataclasses.replace(wm.settings, engine=A.ENGINE_WAVEFRONT)
    # the wavefront's launch parameters for this frame shape (1024 spp, one
    # render of the search), as the renderer would pick them
    from pencil_b200.autotune import autotune
    tune_st = dataclasses.replace(sm_st, samples=32)
    tuned = autotune(ctx, [sm], [tune_st], scene=wm.scene, reps=1, use_cache=False)
    for k in ("queue_capacity", "refill_below", "sort_key", "block_size"):
        setattr(sm_st, k, tuned[k])
    mwin = (0, 0, 256, 256)
    t0 = time.perf_counter()
    mref, mnoise, _ = _reference_image(ctx, sm, sm_st, mwin, frames=32, n=32)
    rec = {"workload": "mesh_box at 256x256, depth 12",
           "reference": "production estimator (quad-light NEE), 32768 spp",
           "reference_seconds": time.perf_counter() - t0,
           "autotuned": {k: tuned[k] for k in ("queue_capacity", "refill_below", "sort_key",
                                                "block_size", "ms")},
           **_equal_rmse_point(ctx, sm, sm_st, mwin, mref, mnoise, max_spp=16384,
                              ref_spp=32768)}
    # the reference's own estimator (no quad light: BSDF sampling only) at
    # 4096 spp against that image
    bs = wm.scene
    bs.lights = [l for l in bs.lights if l.kind != A.LIGHT_QUAD]
    sb = ctx.upload(bs, nodes)
    bimg, bnoise, _ = _reference_image(ctx, sb, sm_st, mwin)
    rec["bsdf_only_4096spp_rel_rmse"] = float(np.sqrt(((bimg - mref) ** 2).mean()) / mref.mean())
    rec["bsdf_only_4096spp_own_noise"] = bnoise
    ctx.free(sb)
    ctx.free(sm)
    out["mesh_box"] = rec
    return out


def measure_bvh_build(ctx, stream) -> dict:
    """Pencil's host SAH build against the device builds -- Pencil's binned
    SAH (the same tree) and an LBVH -- and the render time on each tree
    (wall-clock medians of 5 calls after a first one; the render on the
    sphere cloud with the tuned launch parameters, on the mesh with its
    autotuned ones)."""
    import time

    import torch
    from pencil_b200 import _abi as A
    from pencil_b200 import workloads as W
    out = {}
    for name, wl in (("sphere_cloud", W.sphere_cloud()), ("mesh_box", W.mesh_box())):
        t0 = time.perf_counter()
        host_nodes, host_depth = wl.scene.build_bvh()
        host_ms = (time.perf_counter() - t0) * 1e3
        rec = {"primitives": wl.scene.n_unified, "host_sah_ms": host_ms, "host_depth": host_depth}
        trees = {"sah": host_nodes}
        for method in ("sah", "lbvh"):
            ctx.build_bvh_device(wl.scene, method=method)   # first call loads the module
            times = []
            for _ in range(5):
                t0 = time.perf_counter()
                dev_nodes, dev_depth = ctx.build_bvh_device(wl.scene, method=method)
                times.append((time.perf_counter() - t0) * 1e3)
            rec[f"device_{method}_ms"] = sorted(times)[2]
            rec[f"device_{method}_depth"] = dev_depth
            trees[f"device_{method}"] = dev_nodes
        rec["device_sah_same_nodes"] = float(np.mean(trees["device_sah"] == host_nodes))
        st = wl.settings
        st.engine = A.ENGINE_WAVEFRONT
        if name == "sphere_cloud":
            st.queue_capacity = st.width * st.height * st.samples ** 2
            st.refill_below, st.sort_key = 16, 3
        else:
            st.queue_capacity, st.refill_below, st.sort_key = 1 << 26, 16, 3
        buf = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
        for tree, nodes in trees.items():
            sid = ctx.upload(wl.scene, nodes)
            rec[f"render_ms_{tree}"] = _event_ms(
                stream, lambda: ctx.render_device(sid, st, buf.data_ptr()), 2)
            ctx.free(sid)
        out[name] = rec
    return out


def measure_mesh(ctx, stream) -> dict:
    """The triangle-mesh configuration: a displaced icosphere (8
    subdivisions, 1,310,720 triangles, float32 vertices, int32 indices) in a
    box lit by a 0.25 x 0.25 emissive ceiling quad with next-event
    estimation; 1024x1024, 64 spp, depth 12 (67,108,864 paths per frame).

    Uploaded with Pencil's SAH tree (built at parse time), the wide
    traversals walking a linear BVH over its leaves (PGPU_TRAVERSAL_LBVH,
    built on the device at upload): the renderer's configuration for this
    workload, autotuned, both engines on that tree. The same frame on
    Pencil's own tree (collapsed) is measured beside it with the same
    launch parameters, and the megakernel on Pencil's binary tree."""
    import time

    import torch
    from pencil_b200 import _abi as A
    from pencil_b200 import workloads as W
    from pencil_b200.autotune import autotune
    from pencil_b200.renderer import RenderStats
    wm = W.mesh_box()
    nodes, depth = wm.scene.build_bvh()       # Pencil builds its tree at parse time
    st = wm.settings
    paths = st.width * st.height * st.samples ** 2
    buf = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")

    def frame(sid) -> dict:
        st.engine = A.ENGINE_WAVEFRONT
        wf = _event_ms(stream, lambda: ctx.render_device(sid, st, buf.data_ptr()), 2)
        cnt = RenderStats()
        st.count_rays, st.count_nodes = True, True
        ctx.render(sid, st, stats=cnt)
        st.count_rays, st.count_nodes = False, False
        # device time per kernel class (kernels launched one by one, events
        # around each; outside the timed frames)
        prof = RenderStats()
        st.profile_kernels = True
        ctx.render(sid, st, stats=prof)
        st.profile_kernels = False
        st.engine = A.ENGINE_MEGAKERNEL
        mk = _event_ms(stream, lambda: ctx.render_device(sid, st, buf.data_ptr()), 1)
        st.engine = A.ENGINE_WAVEFRONT
        rays = cnt.extension_rays + cnt.shadow_rays
        return {"wavefront_ms": wf, "wavefront_mpaths_s": paths / wf / 1e3,
                "wavefront_mrays_s": rays / wf / 1e3,
                "megakernel_ms": mk, "megakernel_mpaths_s": paths / mk / 1e3,
                "wavefront_over_megakernel": mk / wf,
                "kernel_ms": {k: round(v, 3) for k, v in prof.kernel_ms.items() if v > 0},
                "ext_node_visits_per_ray": cnt.ext_node_visits / max(1, cnt.extension_rays),
                "shadow_node_visits_per_ray": cnt.shadow_node_visits / max(1, cnt.shadow_rays),
                # leaf records read by leaf tests (48 B per triangle)
                "ext_leaf_bytes_per_ray": cnt.ext_leaf_bytes / max(1, cnt.extension_rays),
                "shadow_leaf_bytes_per_ray": cnt.shadow_leaf_bytes / max(1, cnt.shadow_rays)}

    # the renderer's configuration: LBVH traversal tree over Pencil's leaves
    ctx.set_traversal_tree(A.TRAVERSAL_LBVH)
    try:
        t0 = time.perf_counter()
        sl = ctx.upload(wm.scene, nodes)
        upload_ms = (time.perf_counter() - t0) * 1e3
    finally:
        ctx.set_traversal_tree(A.TRAVERSAL_UPLOADED)
    info = ctx.scene_info(sl)
    # launch parameters from the autotuner (capacity candidates up to 2^26
    # paths: the whole frame in one chunk)
    tuned = autotune(ctx, [sl], [st], scene=wm.scene, reps=1, use_cache=False)
    head = frame(sl)
    ctx.free(sl)
    # Pencil's own tree, collapsed, with the same launch parameters
    t0 = time.perf_counter()
    sm = ctx.upload(wm.scene, nodes)
    upload_pencil_ms = (time.perf_counter() - t0) * 1e3
    pencil = {"tree": "Pencil's SAH tree, collapsed to 4-wide nodes",
              "upload_ms": upload_pencil_ms, "wide_nodes": ctx.scene_info(sm)["n_wide"],
              **frame(sm)}
    st.engine, st.binary_tree = A.ENGINE_MEGAKERNEL, True
    pencil["megakernel_binary_tree_ms"] = _event_ms(
        stream, lambda: ctx.render_device(sm, st, buf.data_ptr()), 1)
    st.engine, st.binary_tree = A.ENGINE_WAVEFRONT, False
    ctx.free(sm)
    return {"workload": "mesh_box: displaced icosphere 1,310,720 triangles in a box, quad-light "
                        "NEE, 1024x1024, 64 spp, depth 12",
            "paths": paths, "triangles": int(len(wm.scene.mesh_indices)),
            "bvh_depth": int(depth),
            "traversal_tree": "linear BVH over Pencil's leaves (their boxes and DFS order: the "
                              "same hits), built on the device at upload",
            "wide_nodes": info["n_wide"], "device_bytes": info["device_bytes"],
            "upload_ms": upload_ms, **head,
            "autotuned": {k: tuned[k] for k in ("queue_capacity", "refill_below", "sort_key",
                                                 "block_size", "ms")},
            "pencil_tree": pencil}


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def run_arena_sizes() -> None:
    """Traversal cost per node visit against scene-arena size: the mesh box
    with icospheres of 6..9 subdivisions (81,920 to 5,242,880 triangles),
    512x512, 64 spp, depth 12, on Pencil's tree collapsed to 4-wide nodes;
    the wavefront with one chunk of 2^24 paths, refill 16, sort key 3,
    64-thread blocks. Per size: the frame on both engines (CUDA events), the
    kernel-class times (events around each class, a second render) and the
    node visits (the counting build), one JSON line each."""
    import torch
    from pencil_b200 import _abi as A
    from pencil_b200 import workloads as W
    from pencil_b200.renderer import GpuContext, RenderStats
    ctx = GpuContext(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    for subdiv in (6, 7, 8, 9):
        wm = W.mesh_box(subdiv=subdiv, width=512, height=512, samples=8, depth=12)
        nodes, _ = wm.scene.build_bvh()
        sid = ctx.upload(wm.scene, nodes)
        info = ctx.scene_info(sid)
        st = wm.settings
        st.engine = A.ENGINE_WAVEFRONT
        st.queue_capacity, st.refill_below, st.sort_key, st.block_size = 1 << 24, 16, 3, 64
        buf = torch.empty((st.height, st.width, 3), dtype=torch.float32, device="cuda")
        wf = _event_ms(stream, lambda: ctx.render_device(sid, st, buf.data_ptr()), 2)
        prof = RenderStats()
        st.profile_kernels = True
        ctx.render(sid, st, stats=prof)
        ctx.render(sid, st, stats=prof)
        st.profile_kernels = False
        cnt = RenderStats()
        st.count_rays, st.count_nodes = True, True
        ctx.render(sid, st, stats=cnt)
        st.count_rays, st.count_nodes = False, False
        st.engine = A.ENGINE_MEGAKERNEL
        mk = _event_ms(stream, lambda: ctx.render_device(sid, st, buf.data_ptr()), 1)
        km = prof.kernel_ms
        print(json.dumps({
            "subdiv": subdiv, "triangles": int(len(wm.scene.mesh_indices)),
            "arena_mb": info["device_bytes"] / 2 ** 20, "wide_nodes": info["n_wide"],
            "ext_visits_per_ray": cnt.ext_node_visits / max(1, cnt.extension_rays),
            "shadow_visits_per_ray": cnt.shadow_node_visits / max(1, cnt.shadow_rays),
            "extend_ms": km["extend"], "shadow_ms": km["shadow"],
            "ps_per_ext_visit": km["extend"] * 1e9 / max(1, cnt.ext_node_visits),
            "ps_per_shadow_visit": km["shadow"] * 1e9 / max(1, cnt.shadow_node_visits),
            "wavefront_ms": wf, "megakernel_ms": mk, "ratio": mk / wf}), flush=True)
        ctx.free(sid)
    ctx.close()


def run_profile_case(args) -> None:
    """One frame of the workload with no CUDA graph, for ncu captures (or one
    adjoint of the box configuration, one device BVH build of the sphere
    cloud, one device tonemap of a 1280x720 frame)."""
    from pencil_b200 import _abi as A
    from pencil_b200 import workloads as W
    from pencil_b200.renderer import GpuContext, RenderStats
    if args.profile_case in ("adjoint", "lbvh", "tonemap"):
        ctx = GpuContext(0)
        if args.profile_case == "adjoint":
            wa, _, _ = W.adjoint_box()
            sid = ctx.upload(wa.scene)
            dl = np.random.default_rng(0).normal(
                size=(wa.settings.height, wa.settings.width, 3)).astype(np.float32)
            st = RenderStats()
            ctx.adjoint(sid, wa.settings, dl, wa.scene.n_materials, len(wa.scene.lights), stats=st)
            out = {"profile_case": "adjoint", "device_ms": st.device_ms}
            ctx.free(sid)
        elif args.profile_case == "lbvh":
            wl = W.sphere_cloud()
            nodes, depth = ctx.build_bvh_device(wl.scene)
            out = {"profile_case": "lbvh", "nodes": int(len(nodes)), "depth": depth}
        else:
            hdr = np.random.default_rng(1).exponential(0.5, (720, 1280, 3)).astype(np.float32)
            px = ctx.tonemap(hdr)
            out = {"profile_case": "tonemap", "bytes": int(px.size)}
        print(json.dumps(out))
        ctx.close()
        return
    mesh = args.profile_case in ("mesh", "mesh_megakernel")
    wl = W.mesh_box() if mesh else W.sphere_cloud()
    st = wl.settings
    st.width //= args.profile_scale
    st.height //= args.profile_scale
    st.use_graph = False
    # the launch parameters the autotuner picks for the workload: one chunk
    # (the whole frame), refill at 16 busy lanes (sphere cloud) or 20 (mesh),
    # shadow work and extension rays sorted by origin cell (sort key 3); the
    # mesh's wide traversals on the LBVH over Pencil's leaves (its bench
    # configuration) unless --profile-pencil-tree
    st.queue_capacity = st.width * st.height * st.samples ** 2
    st.refill_below = 20 if mesh else 16
    st.sort_key = 3
    st.engine = (A.ENGINE_MEGAKERNEL if args.profile_case in ("megakernel", "mesh_megakernel")
                 else A.ENGINE_WAVEFRONT)
    ctx = GpuContext(0)
    if mesh and not args.profile_pencil_tree:
        ctx.set_traversal_tree(A.TRAVERSAL_LBVH)
    sid = ctx.upload(wl.scene, wl.scene.build_bvh()[0] if mesh else None)
    stats = RenderStats()
    img = ctx.render(sid, st, stats=stats)
    assert np.isfinite(img).all()
    out = {"profile_case": args.profile_case, "width": st.width, "height": st.height,
           "launches": stats.kernel_launches, "device_ms": stats.device_ms}
    if args.profile_counts:
        cnt = RenderStats()
        st.count_rays, st.count_nodes = True, True
        ctx.render(sid, st, stats=cnt)
        out.update(extension_rays=cnt.extension_rays, shadow_rays=cnt.shadow_rays,
                   ext_node_visits=cnt.ext_node_visits, shadow_node_visits=cnt.shadow_node_visits)
    print(json.dumps(out))
    ctx.free(sid)
    ctx.close()


def main():
    args = parse_args()
    if args.profile_case:
        run_profile_case(args)
    elif args.arena_sizes:
        run_arena_sizes()
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
