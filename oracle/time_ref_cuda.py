"""Times the reference's own CUDA backend against libfhtgs on the same B200 — MEASUREMENT OF THE
REFERENCE, test infrastructure (oracle/_ref must hold the reference build of oracle/build_ref.sh).

Both sides are called through the same positional drop-in API (`_C_stereo.render`): the
reference's module from oracle/_ref and this package's mirror.  Per call: CUDA events around the
blocking call, 10 warm-up calls, then --calls timed calls; median and p99 in ms, frames/s from the
median.  Also checks that the two produce identical images on the workload.

    python oracle/time_ref_cuda.py [--calls 100] [--n 1000000] [--width 2064 --height 2208]
    python oracle/time_ref_cuda.py --served [--duration 5 --rate 240]
    python oracle/time_ref_cuda.py --plain

--served: the served-stream trace of bench.py --workload served (3 scenes of 0.5M/2M/4M SH3
Gaussians, seeds 1-3, stereo requests of 1440x1584 or 2064x2208 per eye), every request issued
back to back as one blocking `_C_stereo.render` call, through the reference and through this
package's drop-in: requests/s of each (the plain per-request path at saturation).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]


def timed_calls(fn, calls: int, warmup: int = 10):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(calls):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ms.append(a.elapsed_time(b))
    ms = np.asarray(ms)
    return {"median_ms": float(np.median(ms)), "p99_ms": float(np.percentile(ms, 99)),
            "mean_ms": float(ms.mean()), "frames_per_s": float(1000.0 / np.median(ms)), "calls": calls}


def served(a) -> dict:
    import time

    import torch

    import foveatedhtgscudabackend_b200 as F
    from foveatedhtgscudabackend_b200 import scene
    import ref as REF

    sizes = (500_000, 2_000_000, 4_000_000)
    scenes = [F.gaussians_to_torch(scene.make_gaussians(n, 3, seed=i + 1)) for i, n in enumerate(sizes)]
    trace = scene.make_served_requests(a.duration, a.rate, len(scenes), seed=0)
    sts = [[F.settings_from_view(v, K=a.K, active_sh_bases=16) for v in (l, r)] for t, si, l, r in trace]
    ref_mod = REF.module("_C_stereo")
    out = {"workload": f"served trace: {len(trace)} stereo requests, scenes {sizes}, "
                       f"1440x1584 or 2064x2208 per eye (bench.py --workload served, seed 0)"}
    for name, mod in (("reference_cuda", ref_mod), ("ours_dropin", F._C_stereo)):
        for k in range(6):  # warm-up
            si = trace[k][1]
            mod.render(*scenes[si], *sts[k][0].as_tuple(), *sts[k][1].as_tuple(), True, False, False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k, (t, si, l, r) in enumerate(trace):
            mod.render(*scenes[si], *sts[k][0].as_tuple(), *sts[k][1].as_tuple(), True, False, False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out[name] = {"requests_per_s": len(trace) / dt, "seconds": dt}
    out["speedup"] = out["ours_dropin"]["requests_per_s"] / out["reference_cuda"]["requests_per_s"]
    out["gpu"] = torch.cuda.get_device_name()
    return out


def plain(a) -> dict:
    """The plain single-view config (100k SH0 Gaussians, 1280x720, K = 4) through the
    reference's `_C_benchmarking.benchmark` (its foveation cannot be switched off: centred gaze)
    and through this package's drop-in of the same call; images compared."""
    import torch

    import foveatedhtgscudabackend_b200 as F
    from foveatedhtgscudabackend_b200 import scene
    import ref as REF

    g = scene.make_gaussians(100_000, 0, seed=0)
    v = scene.make_view(1280, 720)
    gt = F.gaussians_to_torch(g)
    st = F.settings_from_view(v, K=4, active_sh_bases=1)
    args = (*gt, *st.as_tuple(), True, False, False)
    ref_mod = REF.module("_C_benchmarking")
    mine, theirs = F._C_benchmarking.benchmark(*args), ref_mod.benchmark(*args)
    torch.cuda.synchronize()
    return {"workload": "plain: 100k Gaussians SH0, 1280x720, K=4 (reference layout, centred gaze)",
            "reference_cuda": timed_calls(lambda: ref_mod.benchmark(*args), a.calls),
            "ours_dropin": timed_calls(lambda: F._C_benchmarking.benchmark(*args), a.calls),
            "images_identical": bool(torch.equal(mine, theirs)), "gpu": torch.cuda.get_device_name()}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--calls", type=int, default=100)
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=2064)
    ap.add_argument("--height", type=int, default=2208)
    ap.add_argument("--K", type=int, default=8)
    ap.add_argument("--served", action="store_true")
    ap.add_argument("--plain", action="store_true")
    ap.add_argument("--duration", type=float, default=5.0)
    ap.add_argument("--rate", type=float, default=240.0)
    a = ap.parse_args(argv)
    if a.served:
        print(json.dumps(served(a)))
        return 0
    if a.plain:
        print(json.dumps(plain(a)))
        return 0

    import torch

    import foveatedhtgscudabackend_b200 as F
    from foveatedhtgscudabackend_b200 import scene
    import ref as REF

    g = scene.make_gaussians(a.n, 3, seed=0)
    left, right = scene.make_stereo_views(a.width, a.height, seed=0)
    gt = F.gaussians_to_torch(g)
    st = [F.settings_from_view(v, K=a.K, active_sh_bases=16) for v in (left, right)]
    args = (*gt, *st[0].as_tuple(), *st[1].as_tuple(), True, False, False)
    ref_mod = REF.module("_C_stereo")
    mine = F._C_stereo.render(*args)
    theirs = ref_mod.render(*args)
    torch.cuda.synchronize()
    same = [bool(torch.equal(x, y)) for x, y in zip(mine, theirs)]
    maxabs = [float((x - y).abs().max()) for x, y in zip(mine, theirs)]
    psnr = [float(10 * torch.log10(1.0 / torch.clamp(((x - y).double() ** 2).mean(), min=1e-30))) for x, y in zip(mine, theirs)]
    res = {
        "workload": f"stereo {a.n} Gaussians SH3, 2x{a.width}x{a.height}, K={a.K}",
        "reference_cuda": timed_calls(lambda: ref_mod.render(*args), a.calls),
        "ours_dropin": timed_calls(lambda: F._C_stereo.render(*args), a.calls),
        "images_identical": same, "max_abs": maxabs, "psnr_db": psnr,
        "gpu": torch.cuda.get_device_name(),
    }
    res["speedup_median"] = res["reference_cuda"]["median_ms"] / res["ours_dropin"]["median_ms"]
    print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
