#!/usr/bin/env python
"""Benchmark of the foveated HTGS forward renderer on the stereo foveated workload.

Workload (one "step" = one stereo frame): 1M Gaussians (SH degree 3, seed 0, the synthetic
distributions of foveatedhtgscudabackend_b200.scene), two eyes of 2064x2208 with 63 mm IPD,
gaze at the image centre + N(0, 0.05) NDC, K = 8, fp32, foveation with the reference's
constants (375 px fovea radius, 125 px blend band, 2x-down periphery), fast-math arithmetic
as the reference's _C_stereo module.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  `value` = stereo frames/s of the whole job with the scene
resident in HBM and `--in-flight` frames in flight (default 2: two renderer contexts on two
streams; device time, CUDA events, max over ranks), `single_frame` = the same one frame at a
time; `e2e` = the same through the public C ABI's asynchronous frame with the per-frame
camera/mask inputs copied from pinned host memory and both images copied back to the host
inside the timed region (`dropin_value`: through the blocking drop-in `_C_stereo.render`
instead); `roofline` = the
dominant kernel (full-resolution K-buffer blend) measured live from per-frame CUDA events;
`cpu_baseline` = the host-core restatement of the same algorithm (oracle) on a bounded sample.
Multi-GPU: one process per GPU (torchrun); views are independent, so every rank renders its
own stereo frames of a replicated scene (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "stereo foveated frames/s & p50/p99 latency vs plain path, same B200, PSNR>=50dB"
UNIT = "frames/s"
WORKLOAD = "stereo_foveated_1M_sh3_2x2064x2208_k8"
FP32_LANES_PER_SM = 128
# FP32 operations per (pixel, Gaussian) pair of the reference's blend inner loop up to the
# cutoff test (planes 16, moment 9, direction 9, two dot products 10, compare 1).
FLOP_PER_PAIR = 45


FOVEATION_TEXT = {
    "reference": "reference constants: 375 px fovea radius, 125 px blend band, 2x-down periphery",
    "rings": "rings: full resolution r < {0:g}, 2x down r < {1:g}, 4x down beyond (NDC from the gaze)",
    "none": "none: every tile at full resolution",
}


def ring_samples(view, mode: str, rings) -> np.ndarray:
    """Samples blended per large tile (256, 64 or 16) in the ring / no-foveation modes, from the
    NDC distance of the tile centre to the clamped gaze (the classification of the renderer)."""
    gw, gh = -(-view.width // 16), -(-view.height // 16)
    if mode == "none":
        return np.full(gw * gh, 256, np.int64)
    f32 = np.float32
    gx = min(max(f32(view.gaze_position[0]), f32(0)), f32(view.width - 1))
    gy = min(max(f32(view.gaze_position[1]), f32(0)), f32(view.height - 1))
    tx, ty = np.meshgrid(np.arange(gw), np.arange(gh))
    dx = (f32(16) * tx.astype(f32) + f32(8) - gx) / f32(0.5 * view.width)
    dy = (f32(16) * ty.astype(f32) + f32(8) - gy) / f32(0.5 * view.height)
    r2 = (dx * dx + dy * dy).astype(f32).reshape(-1)
    full, half = f32(rings[0]) * f32(rings[0]), f32(rings[1]) * f32(rings[1])
    return np.where(r2 < full, 256, np.where(r2 < half, 64, 16)).astype(np.int64)


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n-gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=2064)
    ap.add_argument("--height", type=int, default=2208)
    ap.add_argument("--sh-degree", type=int, default=3)
    ap.add_argument("--K", type=int, default=8)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--in-flight", type=int, default=2,
                    help="stereo workload: frames in flight, one renderer context and one stream each "
                         "(1 = one frame at a time; the single-frame numbers are reported either way)")
    ap.add_argument("--blend-split", type=float, default=0.6,
                    help="segment share of the split-blend leg (a tolerance mode); 0 skips the leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--cpu-budget-s", type=float, default=30.0, help="upper bound of the CPU baseline sample")
    ap.add_argument("--workload", choices=["stereo", "batched", "precision", "served", "plain"], default="stereo",
                    help="stereo: the headline stereo frame; batched: 64 mixed-resolution cameras of a 3M scene; "
                         "precision: 6M-Gaussian stereo frame with fp16/bf16 attribute storage; served: a Poisson "
                         "stream of stereo requests against 3 resident scenes through the request server; plain: "
                         "100k SH0 Gaussians, one 1280x720 view, K=4, no foveation")
    ap.add_argument("--n-views", type=int, default=64, help="cameras per batch (batched workload)")
    ap.add_argument("--duration", type=float, default=10.0, help="seconds of arrivals (served workload)")
    ap.add_argument("--rate", type=float, default=240.0, help="request arrivals per second (served workload)")
    ap.add_argument("--rate-sweep", type=float, nargs="*", default=[40.0, 60.0, 80.0, 100.0, 120.0],
                    help="served workload: further Poisson rates (requests/s) replayed for --sweep-duration s each; "
                         "p50/p99 and achieved requests/s per rate (empty: none)")
    ap.add_argument("--sweep-duration", type=float, default=6.0)
    ap.add_argument("--slots", type=int, default=2, help="frames in flight (served workload)")
    ap.add_argument("--max-batch", type=int, default=8, help="requests per frame (served workload)")
    ap.add_argument("--no-plain", action="store_true", help="served workload: skip the plain per-request path")
    ap.add_argument("--served-split", type=float, default=0.0,
                    help="served workload: the server's split-blend segment share (0 = off, bit-identical)")
    ap.add_argument("--foveation", choices=["reference", "rings", "none"], default="reference",
                    help="reference: the reference's fovea/blend/2x layout (comparable with it); rings: full res "
                         "r < --rings[0], 2x down r < --rings[1], 4x down beyond (NDC); none: all full res")
    ap.add_argument("--rings", type=float, nargs=2, default=(0.15, 0.4), help="NDC ring radii (rings foveation)")
    return ap.parse_args(argv)


# ------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------
# DRAM traffic of one blend_kernel<8,8> launch of the headline frame, measured by ncu on B200
# (353.9 MB read + 45.3 MB written; the kernel gathers ~0.95 GB of records, mostly from L2)
BLEND_DRAM_BYTES = 399.2e6


class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples: list[list[str]] = []
        self.skip = 0
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return

        def read():
            for line in self.proc.stdout:
                self.samples.append([x.strip() for x in line.split(",")])
        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()
        # the timed region starts once the sampler is live; samples taken before it are dropped
        t0 = time.time()
        while not self.samples and time.time() - t0 < 3.0 and self.proc.poll() is None:
            time.sleep(0.005)
        self.skip = len(self.samples)

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        timed = self.samples[self.skip:] or self.samples
        for s in timed:
            try:
                sm.append(float(s[0]))
                mx = float(s[1])
                for n, v in zip(names, s[4:8]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------
# workload
# ------------------------------------------------------------------------------------------
def workload(a, rank: int):
    from foveatedhtgscudabackend_b200 import scene
    g = scene.make_gaussians(a.n_gaussians, a.sh_degree, seed=0)
    left, right = scene.make_stereo_views(a.width, a.height, seed=rank)
    return g, left, right


def dist_setup(a):
    from foveatedhtgscudabackend_b200 import dist as D
    if a.impl == "reference":
        return D.world()  # rank 0 alone runs the host-core arm; no process group needed
    return D.init()


def max_over_ranks(x: float, world: int) -> float:
    from foveatedhtgscudabackend_b200 import dist as D
    return D.max_over_ranks(x) if world > 1 else x


def barrier(world: int):
    from foveatedhtgscudabackend_b200 import dist as D
    if world > 1:
        D.barrier()


def cpu_baseline(g, views, a, budget_s: float) -> dict:
    """Host-core restatement of the same algorithm (oracle, FP32, OpenMP), bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # the CPU baseline leg is the one place bench.py runs the oracle
    cores = os.cpu_count() or 1
    fov = dict(foveation=a.foveation, rings=tuple(a.rings))
    t_one, _ = O.time_views(g, [views[0]], n_threads=cores, K=a.K, active_sh_bases=(a.sh_degree + 1) ** 2,
                            precision=32, **fov)
    stages = O.last_stage_seconds()
    sample = "one eye (left) of one stereo frame of the benchmark workload"
    total = t_one
    if 2 * t_one <= budget_s:
        t_two, _ = O.time_views(g, [views[1]], n_threads=cores, K=a.K, active_sh_bases=(a.sh_degree + 1) ** 2,
                                precision=32, **fov)
        stages = {k: v + w for (k, v), w in zip(stages.items(), O.last_stage_seconds().values())}
        total = t_one + t_two
        sample = "one full stereo frame (both eyes) of the benchmark workload"
    else:
        total = 2 * t_one  # second eye extrapolated from the first
        stages = {k: 2 * v for k, v in stages.items()}
    return {"value": 1.0 / total, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": sample, "seconds": round(total, 3),
            "stage_s": {k: round(v, 3) for k, v in stages.items()}}


# ------------------------------------------------------------------------------------------
# our implementation
# ------------------------------------------------------------------------------------------
def split_leg(a, r, gt, st, imgs, stream, world) -> dict:
    """The benchmark frame one at a time with the split blend (a tolerance mode): frame rate,
    stage times, and its images against the default path's (bit-identical to the reference's)."""
    import torch

    exact = [x.clone() for x in imgs]
    r.set_blend_split(a.blend_split, 0)
    try:
        for _ in range(max(a.warmup, 3)):
            r.render(*gt, st, to_chw=True, fast_math=True, images=imgs, sync=True)
        r.set_profiling(True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
        barrier(world)
        torch.cuda.synchronize()
        ev[0].record(stream)
        for k in range(a.steps):
            r.render(*gt, st, to_chw=True, fast_math=True, images=imgs, sync=False)
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
        total = max_over_ranks(ev[0].elapsed_time(ev[a.steps]), world)
        hist = r.stage_history(min(a.steps, 64))
        r.set_profiling(False)
        stats = r.blend_split_stats()
    finally:
        r.set_blend_split(0.0, 0)
    a64 = torch.stack(exact).double()
    b64 = torch.stack(imgs).double()
    d = (a64 - b64).abs()
    mse = float((d * d).mean())
    stages = {k: round(float(np.median([h[k] for h in hist])), 4) for k in hist[0]} if hist else None
    return {"segment_share": a.blend_split, "value": round(world * a.steps / (total / 1000.0), 3),
            "unit": UNIT, "ms_per_step": round(total / a.steps, 4), "stage_ms": stages, **stats,
            "vs_default_path": {"max_abs": float(d.max()), "psnr_db": None if mse == 0 else round(10 * np.log10(1 / mse), 1),
                                "pixels_differing": int((d.amax(dim=1) > 0).sum()),
                                "pixels": int(d[:, 0].numel())},
            "note": "tolerance mode: K-buffer decisions exact, tail sums reordered (max-abs 2e-3 / 50 dB allowed)"}


def run_ours(a, world, rank, local):
    import torch

    import foveatedhtgscudabackend_b200 as F
    from foveatedhtgscudabackend_b200 import _C_stereo

    dev = torch.device("cuda", local)
    g, left, right = workload(a, rank)
    active = (a.sh_degree + 1) ** 2
    gt = F.gaussians_to_torch(g, dev)
    st = [F.settings_from_view(v, K=a.K, active_sh_bases=active, device=dev) for v in (left, right)]
    r = F.Renderer(dev)
    r.set_foveation(a.foveation, *a.rings)
    imgs = [torch.empty((3, v.height, v.width), device=dev) for v in (left, right)]

    # first frame sizes the arena (instance capacity), then warm-up
    r.render(*gt, st, to_chw=True, fast_math=True, images=imgs, sync=True)
    for _ in range(max(a.warmup, 0)):
        r.render(*gt, st, to_chw=True, fast_math=True, images=imgs, sync=True)
    r.set_profiling(True)
    launches0 = r.launch_count()
    stream = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize(dev)
    ev[0].record(stream)
    for k in range(a.steps):
        r.render(*gt, st, to_chw=True, fast_math=True, images=imgs, sync=False)
        ev[k + 1].record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    clk = clocks.stop()
    launches = r.launch_count() - launches0
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(a.steps)]
    total_ms = ev[0].elapsed_time(ev[a.steps])
    info = [r.frame_info(i) for i in range(2)]
    if any(i["overflow"] for i in info):
        raise RuntimeError("instance capacity overflow inside the timed region")
    hist = r.stage_history(min(a.steps, 64))
    r.set_profiling(False)
    digest = image_digest(imgs)  # the benchmark frame's images (the reference arm prints its own)
    total_ms_max = max_over_ranks(total_ms, world)
    value = world * a.steps / (total_ms_max / 1000.0)
    single = {"value": round(value, 3), "ms_per_step": round(total_ms_max / a.steps, 4),
              "latency_ms": {"p50": round(float(np.percentile(step_ms, 50)), 4),
                             "p99": round(float(np.percentile(step_ms, 99)), 4)}}
    split = split_leg(a, r, gt, st, imgs, stream, world) if a.blend_split > 0 else None

    # ---- frames in flight: one context and one stream per frame in flight, frames issued round
    # robin; a frame's kernels fill the SMs that the previous frame's last (densest) tiles leave
    # idle.  Contexts are independent (own arena, own stream), so each frame is the same frame.
    n_fl = max(1, a.in_flight)
    rs, imgs_fl = [r], [imgs]
    streams_fl = [stream] + [torch.cuda.Stream(dev) for _ in range(n_fl - 1)]
    for _ in range(n_fl - 1):
        rr = F.Renderer(dev)
        rr.set_foveation(a.foveation, *a.rings)
        im = [torch.empty((3, v.height, v.width), device=dev) for v in (left, right)]
        for _ in range(1 + max(a.warmup, 0)):
            rr.render(*gt, st, to_chw=True, fast_math=True, images=im, sync=True)
        rs.append(rr)
        imgs_fl.append(im)
    if n_fl > 1:
        launches0 = sum(x.launch_count() for x in rs)
        clocks = ClockSampler(local)
        clocks.start()
        barrier(world)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fs = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
        fe = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
        e0.record(stream)
        for sfl in streams_fl[1:]:
            sfl.wait_event(e0)
        for k in range(a.steps):
            i = k % n_fl
            with torch.cuda.stream(streams_fl[i]):
                fs[k].record(streams_fl[i])
                rs[i].render(*gt, st, to_chw=True, fast_math=True, images=imgs_fl[i], sync=False)
                fe[k].record(streams_fl[i])
        for sfl in streams_fl[1:]:
            stream.wait_stream(sfl)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        clk = clocks.stop()
        launches = sum(x.launch_count() for x in rs) - launches0
        if any(x.frame_info(i)["overflow"] for x in rs for i in range(2)):
            raise RuntimeError("instance capacity overflow inside the timed region")
        step_ms = [fs[k].elapsed_time(fe[k]) for k in range(a.steps)]
        total_ms_max = max_over_ranks(e0.elapsed_time(e1), world)
        value = world * a.steps / (total_ms_max / 1000.0)
        if split is not None:
            # the same frames in flight with the split blend on every context
            for x in rs:
                x.set_blend_split(a.blend_split, 0)
            for i in range(n_fl):
                for _ in range(3):
                    rs[i].render(*gt, st, to_chw=True, fast_math=True, images=imgs_fl[i], sync=True)
            barrier(world)
            torch.cuda.synchronize(dev)
            e0.record(stream)
            for sfl in streams_fl[1:]:
                sfl.wait_event(e0)
            for k in range(a.steps):
                i = k % n_fl
                with torch.cuda.stream(streams_fl[i]):
                    rs[i].render(*gt, st, to_chw=True, fast_math=True, images=imgs_fl[i], sync=False)
            for sfl in streams_fl[1:]:
                stream.wait_stream(sfl)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            barrier(world)
            split_ms = max_over_ranks(e0.elapsed_time(e1), world)
            split["in_flight_value"] = round(world * a.steps / (split_ms / 1000.0), 3)
            split["frames_in_flight"] = n_fl
            for x in rs:
                x.set_blend_split(0.0, 0)

    # ---- dominant kernel: full-resolution blend (fovea + blended tiles), per-frame events ----
    stage_avg = {k: statistics.mean(h[k] for h in hist) for k in hist[0]}
    blend_ms = stage_avg["blend"]
    inter = [r.intermediates(i) for i in range(2)]
    pairs = 0
    for m, view in zip(inter, (left, right)):
        rng = m["instance_ranges"].astype(np.int64)
        cnt = rng[:, 1] - rng[:, 0]
        if a.foveation == "reference":
            # 64 pixels per 8x8 sub-tile (fovea, blended) and 64 samples per periphery tile, as
            # the reference evaluates them
            pairs += 64 * int(cnt[m["tile_index_map_partitioned"]].sum())
        else:
            # samples of each large tile at its ring level x the tile's list length
            pairs += int((ring_samples(view, a.foveation, a.rings) * cnt[0::4]).sum())
    sm_clock = (clk or {}).get("sm_mhz") or 1965.0
    peak_fp32 = torch.cuda.get_device_properties(dev).multi_processor_count * FP32_LANES_PER_SM * 2 * sm_clock * 1e6 / 1e12
    achieved = pairs * FLOP_PER_PAIR / (blend_ms / 1000.0) / 1e12
    if split is not None and split.get("stage_ms"):  # the same work over the split blend's time
        split_achieved = pairs * FLOP_PER_PAIR / (split["stage_ms"]["blend"] / 1000.0) / 1e12
        split["roofline"] = {"achieved": round(split_achieved, 3), "peak": round(peak_fp32, 2), "unit": "TFLOP/s",
                             "frac": round(split_achieved / peak_fp32, 4), "kernel_ms": split["stage_ms"]["blend"],
                             "work": "the default path's reference pair evaluations (see roofline)"}

    # ---- e2e through the public drop-in call with host buffers ----
    # Every step: the per-frame inputs (camera matrices, masks, tables; gaze is a host value)
    # go host->device from pinned memory, the blocking drop-in call renders both eyes, and both
    # images come back device->host into pinned memory.  The copy back of step k runs on a copy
    # stream while step k+1 renders (two pinned output buffers); the timed region ends after the
    # last copy has landed.
    e2e = None
    e2e_steps = 0 if a.no_e2e else (a.e2e_steps or max(3, a.steps))
    # the per-frame inputs of both eyes (camera matrices, masks, area tables) packed into one
    # pinned host buffer, so that each step moves them with a single host->device copy; the
    # settings read device views of the packed copy (gaze stays a host value)
    fields = ("M", "VPM", "VPR_inv", "cam_position", "visibility_mask", "visibility_mask_area_table",
              "fovea_mask_area_table")
    parts, off = [], 0
    for i, s in enumerate(st):
        for f in fields:
            t = getattr(s, f).detach().cpu().contiguous()
            t = t.view(torch.int32) if t.dtype == torch.uint32 else t
            nb = t.numel() * t.element_size()
            parts.append((i, f, t, off, nb))
            off = (off + nb + 15) // 16 * 16
    host_pack = torch.empty(off, dtype=torch.uint8, pin_memory=True)
    for i, f, t, o, nb in parts:
        host_pack[o:o + nb].copy_(t.reshape(-1).view(torch.uint8))
    # one device copy of the packed inputs per context in flight
    dev_packs, sd_packs = [], []
    for _ in range(n_fl):
        dp = torch.empty(off, dtype=torch.uint8, device=dev)
        views_dev = [dict(), dict()]
        for i, f, t, o, nb in parts:
            views_dev[i][f] = dp[o:o + nb].view(t.dtype).view(t.shape)
        dev_packs.append(dp)
        sd_packs.append([s_._replace(**views_dev[i]) for i, s_ in enumerate(st)])
    n_buf = max(2, n_fl)
    out_host = [[torch.empty((3, v.height, v.width), pin_memory=True) for v in (left, right)] for _ in range(n_buf)]
    h2d = int(host_pack.numel()) + 2 * 2 * 4
    d2h = sum(o.numel() * o.element_size() for o in out_host[0])
    copy_stream = torch.cuda.Stream(dev)
    copy_done = [torch.cuda.Event() for _ in range(n_buf)]

    dev_imgs = [[torch.empty((3, v.height, v.width), device=dev) for v in (left, right)] for _ in range(n_buf)]

    def e2e_step(k: int, dropin: bool):
        # asynchronous path: frame k on context k % n_fl and its stream; drop-in: one context
        buf = k % (2 if dropin else n_fl)
        ctx = 0 if dropin else buf
        cur = streams_fl[ctx]
        copy_done[buf].synchronize()  # the copy that used these buffers earlier has landed
        with torch.cuda.stream(cur):
            dev_packs[ctx].copy_(host_pack, non_blocking=True)
            sd = sd_packs[ctx]
            if dropin and a.foveation == "reference":  # the reference's call: blocking, fresh images
                a_img, b_img = _C_stereo.render(*gt, *sd[0].as_tuple(), *sd[1].as_tuple(), True, False, False)
            else:  # the C ABI's asynchronous frame (fhtgs_render_views) into its own images
                a_img, b_img = rs[ctx].render(*gt, sd, to_chw=True, fast_math=True, images=dev_imgs[buf],
                                              sync=dropin)
        copy_stream.wait_stream(cur)
        with torch.cuda.stream(copy_stream):
            out_host[buf][0].copy_(a_img, non_blocking=True)
            out_host[buf][1].copy_(b_img, non_blocking=True)
            a_img.record_stream(copy_stream)
            b_img.record_stream(copy_stream)
            copy_done[buf].record(copy_stream)

    def e2e_run(dropin: bool) -> float:
        for k in range(n_buf):
            e2e_step(k, dropin)
        torch.cuda.synchronize(dev)
        barrier(world)
        t0 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for sfl in streams_fl[1:]:
            sfl.wait_event(t0)
        for k in range(e2e_steps):
            e2e_step(k, dropin)
        stream.wait_stream(copy_stream)
        t1 = torch.cuda.Event(enable_timing=True)
        t1.record(stream)
        torch.cuda.synchronize(dev)
        if any(x.frame_info(i)["overflow"] for x in rs for i in range(2)):
            raise RuntimeError("instance capacity overflow inside the end-to-end region")
        return max_over_ranks(t0.elapsed_time(t1), world)

    if e2e_steps > 0:
        e2e_ms = e2e_run(dropin=False)
        dropin_ms = e2e_run(dropin=True)
        e2e = {"value": round(world * e2e_steps / (e2e_ms / 1000.0), 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "api": "foveatedhtgscudabackend_b200.Renderer.render(sync=False) -> fhtgs_render_views (asynchronous), "
                      f"{n_fl} context(s) on {n_fl} stream(s) in flight",
               "steps": e2e_steps, "h2d": "one packed copy of both eyes' inputs per step",
               "d2h": f"pinned copies on a copy stream, {n_buf} buffers",
               "dropin_value": round(world * e2e_steps / (dropin_ms / 1000.0), 3),
               "dropin_api": "foveatedhtgscudabackend_b200._C_stereo.render (blocking, as the reference's call)"
               if a.foveation == "reference" else "foveatedhtgscudabackend_b200.Renderer.render(sync=True)"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(g, [left, right], a, a.cpu_budget_s)

    if rank != 0:
        return None
    lat = sorted(step_ms)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(total_ms_max / a.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD + ("" if a.foveation == "reference" else f"_{a.foveation}"),
                   "n_gaussians": a.n_gaussians, "sh_degree": a.sh_degree,
                   "views": f"2x{a.width}x{a.height}", "K": a.K, "ipd_m": 0.063,
                   "foveation": FOVEATION_TEXT[a.foveation].format(*a.rings),
                   "math": "fast (matches _C_stereo)", "l2": "inputs larger than L2 (236 MB scene, 2 x 55 MB images)",
                   "parallelism": f"replicated scene, {world} rank(s) x 1 stereo stream, "
                                  f"{max(1, a.in_flight)} frame(s) in flight per rank"},
        "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 4), "p99": round(float(np.percentile(lat, 99)), 4)},
        "frames_in_flight": n_fl,
        "single_frame": single,
        "split_blend": split,
        "e2e": e2e,
        "roofline": {"bound": "fp32", "kernel": "blend_kernel<8> (all tiles of both eyes)",
                     "achieved": round(achieved, 3), "peak": round(peak_fp32, 2), "unit": "TFLOP/s",
                     "frac": round(achieved / peak_fp32, 4),
                     # DRAM bytes of one blend launch on this workload from one ncu capture
                     # (dram__bytes_read.sum + dram__bytes_write.sum): profiles/blend_kernel_stereo_1M_2x2064x2208.md
                     "traffic": BLEND_DRAM_BYTES if a.foveation == "reference" and a.n_gaussians == 1_000_000 else None,
                     "traffic_unit": "bytes per launch (ncu)",
                     "peak_source": "nominal FP32 SIMT: SMs x 128 lanes x 2 x median SM clock under load",
                     "work": f"{pairs} pixel-Gaussian pairs x {FLOP_PER_PAIR} flop "
                             + ("(reference's evaluation count)" if a.foveation == "reference"
                                else "(samples of each tile at its ring level x its list length)"),
                     "kernel_ms": round(blend_ms, 4)},
        "stage_ms": {k: round(v, 4) for k, v in stage_avg.items()},
        "instances_per_eye": [int(i["n_instances"]) for i in info],
        "image_sha256": digest,
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    return line


# ------------------------------------------------------------------------------------------
# plain single view: 100k Gaussians SH0, 1280x720, K = 4, no foveation
# ------------------------------------------------------------------------------------------
def run_plain(a, world, rank, local):
    """100k Gaussians (SH degree 0, seed 0), one 1280x720 view from z = -6, K = 4, no
    foveation (every tile at full resolution; the reference cannot switch its foveation off).
    `value` = frames/s replaying a captured frame graph; beside it the eager frame and one
    blocking drop-in `_C_benchmarking.benchmark` call per frame in the reference's own layout.
    The scene (5.6 MB) and image (11 MB) fit in L2, so L2 is flushed (a 256 MB write) before
    every timed frame and each frame is timed alone; `value` = frames / the sum of frame times."""
    import torch

    import foveatedhtgscudabackend_b200 as F
    from foveatedhtgscudabackend_b200 import _C_benchmarking, scene

    dev = torch.device("cuda", local)
    n = a.n_gaussians if a.n_gaussians != 1_000_000 else 100_000
    g = scene.make_gaussians(n, 0, seed=0)
    v = scene.make_view(1280, 720)
    gt = F.gaussians_to_torch(g, dev)
    st = [F.settings_from_view(v, K=4, active_sh_bases=1, device=dev)]
    stream = torch.cuda.current_stream(dev)
    r = F.Renderer(dev)
    r.set_foveation(a.foveation if a.foveation != "reference" else "none", *a.rings)
    img = [torch.empty((3, v.height, v.width), device=dev)]
    r.render(*gt, st, images=img, sync=True)
    graph = r.capture(*gt, st, images=img, capacity_headroom=1.1)
    steps = max(a.steps, 200)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB of L2

    def timed(fn):
        for _ in range(max(a.warmup, 3)):
            fn()
        barrier(world)
        torch.cuda.synchronize(dev)
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for k in range(steps):
            flush.fill_(k & 255)  # evict the scene and image from L2 before the frame
            e0[k].record(stream)
            fn()
            e1[k].record(stream)
        torch.cuda.synchronize(dev)
        per = sorted(e0[k].elapsed_time(e1[k]) for k in range(steps))
        return max_over_ranks(float(sum(per)), world), per

    launches0 = r.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    graph_ms, per = timed(graph.launch)
    clk = clocks.stop()
    launches = r.launch_count() - launches0
    eager_ms, _ = timed(lambda: r.render(*gt, st, images=img, sync=False))
    graph.close()
    exact = img[0].clone()
    split = None
    split = split_exact = None

    def split_graph(exact_mode: bool) -> dict:
        r.set_blend_split(a.blend_split, 0, exact=exact_mode)
        r.render(*gt, st, images=img, sync=True)
        sgraph = r.capture(*gt, st, images=img, capacity_headroom=1.1)
        split_ms, split_per = timed(sgraph.launch)
        stats = r.blend_split_stats()
        sgraph.close()
        r.set_blend_split(0.0, 0)
        d = (img[0].double() - exact.double()).abs()
        mse = float((d * d).mean())
        return {"segment_share": a.blend_split, "value": round(world * steps / (split_ms / 1000.0), 2),
                "unit": "frames/s", "ms_per_step": round(split_ms / steps, 4),
                "latency_ms": {"p50": round(float(np.percentile(split_per, 50)), 4),
                               "p99": round(float(np.percentile(split_per, 99)), 4)}, **stats,
                "vs_default_path": {"max_abs": float(d.max()),
                                    "psnr_db": None if mse == 0 else round(10 * np.log10(1 / mse), 1)},
                "note": "fragment logs replayed in list order: bit-identical" if exact_mode else
                        "tolerance mode: K-buffer decisions exact, tail sums reordered"}
    if a.blend_split > 0:  # the same frame graph with the split blend, both modes
        split = split_graph(False)
        split_exact = split_graph(True)
    ref_layout_ms, _ = timed(lambda: _C_benchmarking.benchmark(*gt, *st[0].as_tuple(), True, False, False))
    r.close()
    if rank != 0:
        return None
    fov = a.foveation if a.foveation != "reference" else "none"
    return {
        "metric": "plain single-view frames/s (captured frame graph)", "value": round(world * steps / (graph_ms / 1000.0), 2),
        "unit": "frames/s", "n_gpus": world, "steps": steps, "warmup": max(a.warmup, 3),
        "ms_per_step": round(graph_ms / steps, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plain_{n // 1000}k_sh0_1280x720_k4_{fov}", "n_gaussians": n, "sh_degree": 0,
                   "view": "1280x720 from z = -6", "K": 4, "foveation": FOVEATION_TEXT[fov].format(*a.rings),
                   "l2": "L2 flushed (256 MB write) before every timed frame; frames timed one by one"},
        "latency_ms": {"p50": round(float(np.percentile(per, 50)), 4), "p99": round(float(np.percentile(per, 99)), 4)},
        "eager_frames_per_s": round(world * steps / (eager_ms / 1000.0), 2),
        "dropin_reference_layout_frames_per_s": round(world * steps / (ref_layout_ms / 1000.0), 2),
        "split_blend": split,
        "split_blend_exact": split_exact,
        "gpu_launches": int(launches), "clocks": clk,
    }


# ------------------------------------------------------------------------------------------
# batched workload: many cameras of uneven resolution and gaze per frame
# ------------------------------------------------------------------------------------------
def run_batched(a, world, rank, local):
    """64 cameras on a sphere (r in [4, 8]) with resolutions drawn from {640x480, 1280x720,
    1920x1080, 2064x2208} and random gaze, of one 3M-Gaussian SH3 scene, K = 8.  Three ways:
    the batch as one captured frame graph after autotuning (`value`), the batch as one eager
    frame, and the plain per-request path (each view through the blocking drop-in
    `_C_benchmarking.benchmark`, one call per view)."""
    import torch

    import foveatedhtgscudabackend_b200 as F
    from foveatedhtgscudabackend_b200 import _C_benchmarking, scene

    dev = torch.device("cuda", local)
    n_gauss = a.n_gaussians if a.n_gaussians != 1_000_000 else 3_000_000
    g = scene.make_gaussians(n_gauss, a.sh_degree, seed=0)
    views = scene.make_batched_views(a.n_views, seed=rank)
    active = (a.sh_degree + 1) ** 2
    gt = F.gaussians_to_torch(g, dev)
    st = [F.settings_from_view(v, K=a.K, active_sh_bases=active, device=dev) for v in views]
    pixels = sum(v.width * v.height for v in views)
    stream = torch.cuda.current_stream(dev)

    def timed(fn, steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        barrier(world)
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        for k in range(steps):
            fn()
            ev[k + 1].record(stream)
        torch.cuda.synchronize(dev)
        per = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
        return max_over_ranks(ev[0].elapsed_time(ev[steps]), world), per

    # per view 1-3 foveation regions (seeded): 1 = every tile at full resolution; 2 = full
    # resolution within NDC radius 0.15 of the gaze, 2x down beyond; 3 = full / 2x within 0.4 /
    # 4x beyond (the rings of the stereo config)
    rng = np.random.default_rng(rank + 4242)
    rings = [int(x) for x in rng.integers(1, 4, size=len(views))]
    vf = [{1: "none", 2: ("rings", 0.15, 100.0), 3: ("rings", 0.15, 0.4)}[c] for c in rings]
    r = F.Renderer(dev)
    imgs = [torch.empty((3, v.height, v.width), device=dev) for v in views]
    r.render(*gt, st, images=imgs, sync=True, view_foveation=vf)
    tuning = r.autotune(*gt, st, repeats=2, view_foveation=vf)
    graph = r.capture(*gt, st, images=imgs, capacity_headroom=1.1, view_foveation=vf)
    for _ in range(max(a.warmup, 0)):
        graph.launch()
    launches0 = r.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    graph_ms, graph_per = timed(graph.launch, a.steps)
    clk = clocks.stop()
    launches = r.launch_count() - launches0
    overflow = any(r.frame_info(i)["overflow"] for i in range(len(st)))
    eager_ms, _ = timed(lambda: r.render(*gt, st, images=imgs, sync=False, view_foveation=vf), a.steps)
    graph.close()
    split = None
    if a.blend_split > 0:  # the same batch graph with the split blend (tolerance mode)
        exact = [x.clone() for x in imgs]
        r.set_blend_split(a.blend_split, 0)
        r.render(*gt, st, images=imgs, sync=True, view_foveation=vf)
        sgraph = r.capture(*gt, st, images=imgs, capacity_headroom=1.1, view_foveation=vf)
        for _ in range(max(a.warmup, 0)):
            sgraph.launch()
        split_ms, _ = timed(sgraph.launch, a.steps)
        stats = r.blend_split_stats()
        sgraph.close()
        r.set_blend_split(0.0, 0)
        dmax = max(float((x.double() - y.double()).abs().max()) for x, y in zip(imgs, exact))
        split = {"segment_share": a.blend_split, "value": round(world * a.steps * len(st) / (split_ms / 1000.0), 2),
                 "unit": "views/s", "ms_per_step": round(split_ms / a.steps, 3), **stats,
                 "vs_default_path_max_abs": dmax,
                 "note": "tolerance mode: K-buffer decisions exact, tail sums reordered"}
    # plain per-request path: one blocking call per view, each with its own foveation
    rp = F.Renderer(dev)
    plain_steps = max(1, min(a.steps, 3))

    def plain_frame():
        for s_, f_ in zip(st, vf):
            rp.render(*gt, [s_], sync=True, view_foveation=[f_])
    plain_frame()
    plain_ms, _ = timed(plain_frame, plain_steps)
    rp.close()
    r.close()
    if rank != 0:
        return None
    nv = len(st)
    lat = sorted(graph_per)
    return {
        "metric": "batched views/s (mixed-resolution cameras, one captured frame graph per batch)",
        "value": round(world * a.steps * nv / (graph_ms / 1000.0), 2), "unit": "views/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(graph_ms / a.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batched_{nv}views_{n_gauss // 1000}k_sh{a.sh_degree}_k{a.K}", "n_gaussians": n_gauss,
                   "views": nv, "megapixels_per_batch": round(pixels / 1e6, 2),
                   "resolutions": "uniform from 640x480, 1280x720, 1920x1080, 2064x2208",
                   "cameras": "sphere r in [4, 8] looking at the origin, gaze uniform in [-0.8, 0.8]^2 NDC",
                   "foveation": "per view 1-3 regions: all full / full r<0.15 + 2x / full r<0.15, 2x r<0.4, 4x "
                                "(seeded; counts per view in `view_regions`)",
                   "l2": "inputs larger than L2"},
        "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3), "p99": round(float(np.percentile(lat, 99)), 3)},
        "eager_batch_views_per_s": round(world * a.steps * nv / (eager_ms / 1000.0), 2),
        "plain_per_view_views_per_s": round(world * plain_steps * nv / (plain_ms / 1000.0), 2),
        "plain_per_view_api": "Renderer.render(sync=True), one blocking call per view (the drop-in has only the reference's foveation)",
        "view_regions": rings,
        "tuning": tuning, "overflow": overflow, "split_blend": split, "gpu_launches": int(launches), "clocks": clk,
    }


# ------------------------------------------------------------------------------------------
# reduced-precision storage workload
# ------------------------------------------------------------------------------------------
def run_precision(a, world, rank, local):
    """6M Gaussians SH3, stereo 2 x 2064x2208, K = 8: the scene stored as fp32 and as the
    reduced-precision format (positions fp32; scales, quaternions, opacities fp16; SH bf16;
    fp32 arithmetic).  `value` = frames/s of the reduced-precision scene; beside it the fp32
    scene's frames/s and the image error of the one against the other (PSNR, max-abs)."""
    import torch

    import foveatedhtgscudabackend_b200 as F
    from foveatedhtgscudabackend_b200 import scene

    dev = torch.device("cuda", local)
    n_gauss = a.n_gaussians if a.n_gaussians != 1_000_000 else 6_000_000
    g = scene.make_gaussians(n_gauss, a.sh_degree, seed=0)
    left, right = scene.make_stereo_views(a.width, a.height, seed=rank)
    active = (a.sh_degree + 1) ** 2
    st = [F.settings_from_view(v, K=a.K, active_sh_bases=active, device=dev) for v in (left, right)]
    full = F.gaussians_to_torch(g, dev)
    half = F.to_half_storage(*full)
    bytes_full = sum(t.numel() * t.element_size() for t in full)
    bytes_half = sum(t.numel() * t.element_size() for t in half)
    del g
    stream = torch.cuda.current_stream(dev)
    out = {}
    for name, gt in (("fp32", full), ("half", half)):
        r = F.Renderer(dev)
        imgs = [torch.empty((3, v.height, v.width), device=dev) for v in (left, right)]
        r.render(*gt, st, images=imgs, sync=True)
        for _ in range(max(a.warmup, 0)):
            r.render(*gt, st, images=imgs, sync=False)
        r.set_profiling(True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
        clocks = ClockSampler(local) if name == "half" else None
        if clocks:
            clocks.start()
        barrier(world)
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        launches0 = r.launch_count()
        for k in range(a.steps):
            r.render(*gt, st, images=imgs, sync=False)
            ev[k + 1].record(stream)
        torch.cuda.synchronize(dev)
        launches = r.launch_count() - launches0
        clk = clocks.stop() if clocks else None
        total = max_over_ranks(ev[0].elapsed_time(ev[a.steps]), world)
        per = sorted(ev[k].elapsed_time(ev[k + 1]) for k in range(a.steps))
        hist = r.stage_history(min(a.steps, 64))
        overflow = any(r.frame_info(i)["overflow"] for i in range(2))
        out[name] = dict(fps=world * a.steps / (total / 1000.0), p50=float(np.percentile(per, 50)),
                         p99=float(np.percentile(per, 99)), images=[x.clone() for x in imgs],
                         stages={k: round(statistics.mean(h[k] for h in hist), 4) for k in hist[0]},
                         launches=launches, clk=clk, overflow=overflow)
        r.close()
    err = []
    for x, y in zip(out["half"]["images"], out["fp32"]["images"]):
        mse = float(((x.double() - y.double()) ** 2).mean())
        err.append({"psnr_db": round(10 * np.log10(1.0 / mse), 2) if mse > 0 else float("inf"),
                    "max_abs": round(float((x - y).abs().max()), 5)})
    if rank != 0:
        return None
    h, f = out["half"], out["fp32"]
    return {
        "metric": "stereo frames/s with fp16/bf16 Gaussian storage (fp32 arithmetic)", "value": round(h["fps"], 3),
        "unit": "frames/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(1000.0 / h["fps"] * world, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16/bf16 storage, f32 compute", "data": "synthetic",
        "config": {"workload": f"precision_stereo_{n_gauss // 1000}k_sh{a.sh_degree}_2x{a.width}x{a.height}_k{a.K}",
                   "n_gaussians": n_gauss, "storage": "positions fp32; scales, rotations, opacities fp16; SH bf16",
                   "scene_bytes": {"fp32": bytes_full, "half": bytes_half},
                   "foveation": "reference constants", "l2": "inputs larger than L2"},
        "latency_ms": {"p50": round(h["p50"], 4), "p99": round(h["p99"], 4)},
        "fp32_storage": {"frames_per_s": round(f["fps"], 3), "p50_ms": round(f["p50"], 4), "stage_ms": f["stages"]},
        "stage_ms": h["stages"],
        "error_vs_fp32_storage": err,
        "gpu_launches": int(h["launches"]), "overflow": h["overflow"] or f["overflow"], "clocks": h["clk"],
    }


# ------------------------------------------------------------------------------------------
# served stream: resident scenes, Poisson arrivals, continuous batching vs one call per request
# ------------------------------------------------------------------------------------------
SERVED_SCENES = (500_000, 2_000_000, 4_000_000)


def run_served(a, world, rank, local):
    """3 resident scenes (0.5M, 2M, 4M Gaussians, SH3, seeds 1-3); stereo requests arriving
    Poisson at `--rate` per second for `--duration` s, each with a uniformly drawn scene, one
    resolution per request from {1440x1584, 2064x2208} per eye, a random head pose (sphere,
    r in [4, 8]) and gaze; K = 8, fast-math, 150 GB budget.  The same trace runs through
    (a) the request server (continuous batching over `--slots` frames in flight) — `value`,
    and (b) the plain per-request path: one blocking drop-in `_C_stereo.render` call per
    request, in arrival order.  Latency = GPU completion - scheduled arrival.  Both paths
    also drain the whole trace submitted at once (saturated requests/s)."""
    import torch

    import foveatedhtgscudabackend_b200 as F
    from foveatedhtgscudabackend_b200 import _C_stereo, scene
    from foveatedhtgscudabackend_b200.serving import Server

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    scenes = [F.gaussians_to_torch(scene.make_gaussians(n, a.sh_degree, seed=i + 1), dev)
              for i, n in enumerate(SERVED_SCENES)]
    active = (a.sh_degree + 1) ** 2
    trace = scene.make_served_requests(a.duration, a.rate, len(scenes), seed=rank)
    warm = scene.make_served_requests(1.0, 96.0, len(scenes), seed=1000 + rank)
    n_req = len(trace)

    srv = Server(dev, hbm_budget_bytes=150e9, max_in_flight=a.slots, max_batch_requests=a.max_batch,
                 blend_split=a.served_split)
    ids = [srv.add_scene(*gt, K=a.K, active_sh_bases=active, foveation=a.foveation, rings=tuple(a.rings))
           for gt in scenes]

    def drain_all(expect):
        got = 0
        idle = 0
        while got < expect:
            cs = srv.poll(max_completions=256, wait_ms=1000)
            idle = 0 if cs else idle + 1
            if idle >= 60:  # frames of many large views take seconds; a minute without any is a fault
                raise RuntimeError("server made no progress for 60 s")
            for c in cs:
                if not c.ok:
                    raise RuntimeError(f"request failed: {c.message}")
                srv.release(c.ticket)
                got += 1
        return got

    # warm-up (untimed): full-size frames of every scene size the slot arenas and output pool
    for rep in range(2):
        srv.pause()
        for t, si, l, r in warm:
            srv.submit(ids[si], [l, r])
        srv.resume()
        drain_all(len(warm))

    def replay(tr, prep):
        """Poisson replay of a trace through the server: latency (GPU completion - scheduled
        arrival) per request, seconds from the first arrival to the last completion, and the
        views of the frame that rendered each request."""
        n = len(tr)
        t0 = srv.clock_ms() + 20.0
        arrive = [t0 + 1000.0 * t for t, *_ in tr]
        lat = [0.0] * n
        fviews = []
        i = done = 0
        last = t0
        while done < n:
            now = srv.clock_ms()
            while i < n and arrive[i] <= now:
                srv.submit_prepared(prep[i])
                i += 1
            wait = int(min(max(arrive[i] - srv.clock_ms() - 1.0, 0.0), 5.0)) if i < n else 5
            for c in srv.poll(max_completions=256, wait_ms=wait):
                if not c.ok:
                    raise RuntimeError(f"request failed: {c.message}")
                lat[c.tag] = c.done_ms - arrive[c.tag]
                last = max(last, c.done_ms)
                fviews.append(c.frame_views)
                srv.release(c.ticket)
                done += 1
        return lat, (last - t0) / 1000.0, fviews

    # latency floor: each scene and resolution served alone, one request at a time (median of 5)
    alone = {}
    for si in range(len(scenes)):
        for (t, si_, l, r) in warm:
            key = f"{SERVED_SCENES[si]}@{l.width}x{l.height}"
            if key in alone:
                continue
            lat1 = []
            for _ in range(5):
                tk = srv.submit(ids[si], [l, r])
                c = []
                while not c:
                    c = srv.poll(max_completions=1, wait_ms=1000)
                lat1.append(c[0].done_ms - c[0].submit_ms)
                srv.release(c[0].ticket)
            alone[key] = round(float(np.median(lat1)), 3)
            if len(alone) == 2 * (si + 1):
                break

    prepared = [srv.prepare(ids[si], [l, r], tag=k) for k, (t, si, l, r) in enumerate(trace)]
    stats0 = srv.stats()
    clocks = ClockSampler(local)
    clocks.start()
    # (a) server, Poisson replay
    lat_s, served_s, frame_views = replay(trace, prepared)
    stats1 = srv.stats()
    # saturated: the whole trace at once
    srv.pause()
    ts = srv.clock_ms()
    for p in prepared:
        srv.submit_prepared(p)
    srv.resume()
    got = 0
    sat_done = ts
    while got < n_req:
        for c in srv.poll(max_completions=256, wait_ms=1000):
            sat_done = max(sat_done, c.done_ms)
            srv.release(c.ticket)
            got += 1
    served_sat = n_req / ((sat_done - ts) / 1000.0)
    clk = clocks.stop()
    # rate sweep: the same server at further Poisson rates (each its own seeded trace)
    pct = lambda x, q: round(float(np.percentile(x, q)), 3)
    sweep = []
    for rate in a.rate_sweep:
        tr = scene.make_served_requests(a.sweep_duration, rate, len(scenes), seed=2000 + int(rate) + rank)
        prep = [srv.prepare(ids[si], [l, r], tag=k) for k, (t, si, l, r) in enumerate(tr)]
        lat, secs, fv = replay(tr, prep)
        by_scene = {}
        for k, (t, si, l, r) in enumerate(tr):
            by_scene.setdefault(SERVED_SCENES[si], []).append(lat[k])
        achieved = len(tr) / secs
        offered = len(tr) / max(tr[-1][0], 1e-9) if tr else 0.0  # this trace's own arrival rate
        sweep.append({"rate_per_s": rate, "requests": len(tr), "offered_per_s": round(offered, 2),
                      "achieved_per_s": round(achieved, 2),
                      # keeps up: completions follow the arrivals (within 5 %) and the last
                      # request did not wait a whole second longer than the median one
                      "keeps_up": bool(achieved >= 0.95 * offered and max(lat) < np.median(lat) + 1000.0), "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                      "p99_ms_by_scene": {str(n): pct(x, 99) for n, x in sorted(by_scene.items())},
                      "mean_frame_views": round(float(np.mean(fv)), 2)})
    srv.close()

    # (b) plain per-request path on the same trace (device settings prepared beforehand)
    plain = None
    if not a.no_plain:
        if a.foveation == "reference":
            def plain_call(si, sd):
                return _C_stereo.render(*scenes[si], *sd[0].as_tuple(), *sd[1].as_tuple(), True, False, False)
        else:  # the drop-in call has only the reference's foveation: a blocking Renderer call
            rp = F.Renderer(dev)
            rp.set_foveation(a.foveation, *a.rings)

            def plain_call(si, sd):
                return rp.render(*scenes[si], sd, to_chw=True, fast_math=True, sync=True)
        sts = [[F.settings_from_view(v, K=a.K, active_sh_bases=active, device=dev) for v in (l, r)]
               for t, si, l, r in trace]
        for t, si, l, r in warm[:6]:
            w = [F.settings_from_view(v, K=a.K, active_sh_bases=active, device=dev) for v in (l, r)]
            plain_call(si, w)
        torch.cuda.synchronize(dev)
        clock = time.perf_counter
        t0p = 1000.0 * clock() + 20.0
        lat_p = []
        for k, (t, si, l, r) in enumerate(trace):
            arr = t0p + 1000.0 * t
            while 1000.0 * clock() < arr:
                pass
            plain_call(si, sts[k])
            lat_p.append(1000.0 * clock() - arr)
        plain_s = (1000.0 * clock() - t0p) / 1000.0
        ts = clock()
        for k, (t, si, l, r) in enumerate(trace):
            plain_call(si, sts[k])
        plain_sat = n_req / (clock() - ts)
        plain = {"api": ("foveatedhtgscudabackend_b200._C_stereo.render" if a.foveation == "reference"
                         else "foveatedhtgscudabackend_b200.Renderer.render (blocking)") + ", one call per request",
                 "requests_per_s": round(n_req / plain_s, 2), "p50_ms": pct(lat_p, 50), "p99_ms": pct(lat_p, 99),
                 "max_ms": round(max(lat_p), 3), "saturated_requests_per_s": round(plain_sat, 2)}

    if rank != 0:
        return None
    return {
        "metric": "served stereo requests/s & p50/p99 latency vs plain per-request path (Poisson arrivals)",
        "value": round(n_req / served_s, 2), "unit": "requests/s", "n_gpus": world, "steps": n_req, "warmup": 2 * len(warm),
        "ms_per_step": round(1000.0 * served_s / n_req, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"served_{'_'.join(str(n // 1000) + 'k' for n in SERVED_SCENES)}_sh{a.sh_degree}_poisson{a.rate:g}"
                               + ("" if a.foveation == "reference" else f"_{a.foveation}"),
                   "foveation": FOVEATION_TEXT[a.foveation].format(*a.rings),
                   "scenes": list(SERVED_SCENES), "rate_per_s": a.rate, "duration_s": a.duration, "requests": n_req,
                   "resolutions_per_eye": "uniform from 1440x1584, 2064x2208", "K": a.K,
                   "head_pose": "sphere r in [4, 8] looking at the origin; gaze N(0, 0.1) NDC",
                   "hbm_budget_gb": 150, "slots": a.slots, "max_batch_requests": a.max_batch,
                   "blend_split": a.served_split or "off (bit-identical)",
                   "l2": "inputs larger than L2"},
        "latency_ms": {"p50": pct(lat_s, 50), "p99": pct(lat_s, 99), "max": round(max(lat_s), 3)},
        "plain_path": plain,
        "saturated_requests_per_s": round(served_sat, 2),
        "throughput_vs_plain": round((n_req / served_s) / plain["requests_per_s"], 3) if plain else None,
        "saturated_vs_plain": round(served_sat / plain["saturated_requests_per_s"], 3) if plain else None,
        "mean_frame_views": round(float(np.mean(frame_views)), 2),
        "alone_latency_ms": alone,
        "rate_sweep": sweep,
        "highest_sustained_rate_per_s": max([x["rate_per_s"] for x in sweep if x["keeps_up"]], default=None),
        "server": {k: stats1[k] - stats0.get(k, 0) if k in ("frames", "views", "retries", "admission_waits") else stats1[k]
                   for k in ("frames", "views", "retries", "admission_waits", "peak_resident_bytes", "max_frame_requests")},
        "clocks": clk,
    }


# ------------------------------------------------------------------------------------------
# reference arm: the reference algorithm on the host cores
# ------------------------------------------------------------------------------------------
def image_digest(imgs) -> list[str]:
    """SHA-256 of each image's float32 bytes (the same frame in both arms gives the same digest
    exactly when the images are bit-identical)."""
    import hashlib
    return [hashlib.sha256(t.detach().contiguous().cpu().numpy().tobytes()).hexdigest() for t in imgs]


def reference_cuda_leg(a, g, left, right, calls: int, warmup: int = 10) -> dict:
    """The reference's own CUDA backend on this GPU: `_C_stereo.render` of the reference, built
    from its sources with its own flags (+ sm_100a) into oracle/_ref, called through its pybind
    API on the benchmark frame.  Device leg: CUDA events around each blocking call, `warmup`
    untimed calls, then `calls` timed calls; frames/s from the median.  End-to-end leg: per call
    the per-frame inputs of both eyes (one packed pinned host->device copy) and both images back
    to pinned host memory, as the drop-in leg of our arm.  After the timed regions the frame is
    rendered once by this package's drop-in and the images are compared."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref as REF  # the reference arm may load the reference build under oracle/_ref
    import foveatedhtgscudabackend_b200 as F

    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    try:
        mod = REF.module("_C_stereo")
    except ImportError as exc:
        return {"unavailable": f"reference build not found under oracle/_ref ({exc})"}
    dev = torch.device("cuda", torch.cuda.current_device())
    gt = F.gaussians_to_torch(g, dev)
    st = [F.settings_from_view(v, K=a.K, active_sh_bases=(a.sh_degree + 1) ** 2, device=dev) for v in (left, right)]
    args = (*gt, *st[0].as_tuple(), *st[1].as_tuple(), True, False, False)
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        mod.render(*args)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev.index)
    clocks.start()
    ms = []
    for _ in range(calls):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mod.render(*args)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    clk = clocks.stop()

    # end to end: the same per-frame copies as our drop-in leg (packed inputs in, images out)
    fields = ("M", "VPM", "VPR_inv", "cam_position", "visibility_mask", "visibility_mask_area_table",
              "fovea_mask_area_table")
    parts, off = [], 0
    for i, s_ in enumerate(st):
        for f in fields:
            t = getattr(s_, f).detach().cpu().contiguous()
            t = t.view(torch.int32) if t.dtype == torch.uint32 else t
            nb = t.numel() * t.element_size()
            parts.append((i, f, t, off, nb))
            off = (off + nb + 15) // 16 * 16
    host_pack = torch.empty(off, dtype=torch.uint8, pin_memory=True)
    for i, f, t, o, nb in parts:
        host_pack[o:o + nb].copy_(t.reshape(-1).view(torch.uint8))
    dev_pack = torch.empty(off, dtype=torch.uint8, device=dev)
    views_dev = [dict(), dict()]
    for i, f, t, o, nb in parts:
        dt = torch.uint32 if getattr(st[i], f).dtype == torch.uint32 else t.dtype
        views_dev[i][f] = dev_pack[o:o + nb].view(t.dtype).view(t.shape).view(dt)
    sd = [s_._replace(**views_dev[i]) for i, s_ in enumerate(st)]
    out_host = [[torch.empty((3, v.height, v.width), pin_memory=True) for v in (left, right)] for _ in range(2)]
    copy_stream = torch.cuda.Stream(dev)
    copy_done = [torch.cuda.Event() for _ in range(2)]

    def e2e_step(k):
        buf = k % 2
        copy_done[buf].synchronize()
        dev_pack.copy_(host_pack, non_blocking=True)
        li, ri = mod.render(*gt, *sd[0].as_tuple(), *sd[1].as_tuple(), True, False, False)
        copy_stream.wait_stream(stream)
        with torch.cuda.stream(copy_stream):
            out_host[buf][0].copy_(li, non_blocking=True)
            out_host[buf][1].copy_(ri, non_blocking=True)
            li.record_stream(copy_stream)
            ri.record_stream(copy_stream)
            copy_done[buf].record(copy_stream)

    for k in range(2):
        e2e_step(k)
    torch.cuda.synchronize(dev)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(calls):
        e2e_step(k)
    stream.wait_stream(copy_stream)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = t0.elapsed_time(t1)

    theirs = mod.render(*args)
    mine = F._C_stereo.render(*args)  # compared after the timed regions only
    torch.cuda.synchronize(dev)
    same = [bool(torch.equal(x, y)) for x, y in zip(mine, theirs)]
    maxabs = [float((x - y).abs().max()) for x, y in zip(mine, theirs)]
    psnr = [float(10 * torch.log10(1.0 / torch.clamp(((x - y).double() ** 2).mean(), min=1e-30)))
            for x, y in zip(mine, theirs)]
    ms_sorted = np.asarray(ms)
    med = float(np.median(ms_sorted))
    return {
        "value": round(1000.0 / med, 3), "unit": UNIT,
        "api": "oracle/_ref FoveatedHTGSCudaBackend._C_stereo.render (the reference's pybind module, built from its "
               "sources by oracle/build_ref.sh with its own flags + sm_100a), blocking call per frame",
        "ms": {"median": round(med, 4), "p50": round(float(np.percentile(ms_sorted, 50)), 4),
               "p99": round(float(np.percentile(ms_sorted, 99)), 4), "mean": round(float(ms_sorted.mean()), 4)},
        "calls": calls, "warmup_calls": warmup,
        "e2e": {"value": round(calls / (e2e_ms / 1000.0), 3), "unit": UNIT,
                "h2d_bytes_per_step": int(host_pack.numel()), "d2h_bytes_per_step":
                    int(sum(o.numel() * o.element_size() for o in out_host[0])),
                "note": "one packed pinned copy of both eyes' per-frame inputs in, both images out on a copy "
                        "stream (2 pinned buffers), as the drop-in leg of our arm"},
        "clocks": clk,
        "image_sha256": image_digest(theirs),
        "images_identical_to_ours": same, "max_abs_vs_ours": maxabs, "psnr_db_vs_ours": psnr,
    }


def run_reference(a, world, rank):
    if rank != 0:
        return None
    g, left, right = workload(a, 0)
    cpu = cpu_baseline(g, [left, right], a, a.cpu_budget_s)
    # each step is the bounded sample above; K steps repeat it only when it is short
    per = 1.0 / cpu["value"]
    steps = 1 if per > 5.0 else max(1, min(a.steps, int(30.0 / max(per, 1e-3))))
    ref_cuda = reference_cuda_leg(a, g, left, right, calls=max(100, a.steps))
    return {
        "metric": METRIC, "impl": "reference", "value": round(cpu["value"], 5), "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": 0, "ms_per_step": round(per * 1000.0, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_gaussians": a.n_gaussians, "views": f"2x{a.width}x{a.height}", "K": a.K,
                   "steps_note": f"host-core leg: {steps} step(s) of one full stereo frame each (seconds per frame on "
                                 "the host cores), no warm-up; --steps/--warmup apply to our arm. reference_cuda leg: "
                                 f"10 warm-up calls, then {max(100, a.steps)} timed calls",
                   "l2": "inputs larger than L2 (236 MB scene, 2 x 55 MB images)"},
        "cpu_baseline": cpu,
        "e2e": {"value": round(cpu["value"], 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": ref_cuda,
        "note": "value: the reference has no CPU path; this is the host-core restatement of its algorithm (oracle/). "
                "reference_cuda: the reference's own CUDA backend on the same GPU and frame",
    }


def main(argv=None) -> int:
    a = parse(argv)
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # not under a launcher: start the --gpus ranks here (one process per GPU, torchrun on
        # 127.0.0.1); each rank runs this script with the same arguments
        from foveatedhtgscudabackend_b200 import dist as D
        return D.launch_ranks(a.gpus, [os.path.abspath(__file__)] + list(sys.argv[1:] if argv is None else argv))
    world, rank, local = dist_setup(a)
    if world != a.gpus:
        raise SystemExit(f"bench.py: --gpus {a.gpus} but {world} rank(s) were started")
    try:
        if a.impl == "reference":
            line = run_reference(a, world, rank)
        elif a.workload == "batched":
            line = run_batched(a, world, rank, local)
        elif a.workload == "precision":
            line = run_precision(a, world, rank, local)
        elif a.workload == "served":
            line = run_served(a, world, rank, local)
        elif a.workload == "plain":
            line = run_plain(a, world, rank, local)
        else:
            line = run_ours(a, world, rank, local)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1 and a.impl == "ours":
            from foveatedhtgscudabackend_b200 import dist as D
            D.finalize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
