"""Generates the golden fixtures under tests/golden/ from the REFERENCE implementation.

Runs on a machine with a B200 and the reference built by `oracle/build_ref.sh` and
`make -C oracle harness` (both under oracle/_ref/).  For each case below it regenerates the
seeded synthetic inputs (foveatedhtgscudabackend_b200.scene), runs

  * the reference's own kernels through oracle/ref_harness.cu (every intermediate), and
  * the reference's pybind module (_C.render / _C_benchmarking.benchmark / _C_stereo.render)
    for the final image(s),

and stores the results as compressed .npz files.  Inputs are not stored: they are rebuilt from
the case parameters (the generator is deterministic), see `case_inputs`.

    python tests/golden/make_golden.py --out tests/golden
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from foveatedhtgscudabackend_b200 import scene  # noqa: E402

# Each case: scene + camera(s) + settings + which reference entry point produces the image.
CASES = {
    "mono_ieee_masked_blur_shbg": dict(
        module="_C", n=8000, sh_degree=3, seed=11, views=[dict(w=640, h=480, gaze=[120.0, 100.0], mask_p=0.85,
                                                               mask_seed=5)],
        K=8, active_sh=16, background=1, blur=True, to_chw=True, aaa=False),
    "mono_ieee_aaa_hwc": dict(
        module="_C", n=8000, sh_degree=3, seed=12, views=[dict(w=640, h=480, gaze=[520.0, 90.0])],
        K=4, active_sh=9, background=0, blur=False, to_chw=False, aaa=True),
    "mono_fast_texraw_k16": dict(
        module="_C_benchmarking", n=8000, sh_degree=1, seed=13, views=[dict(w=640, h=480, gaze=[600.0, 450.0])],
        K=16, active_sh=4, background=3, blur=False, to_chw=True, aaa=False),
    "mono_fast_plain_720p_sh0": dict(
        module="_C_benchmarking", n=20000, sh_degree=0, seed=0, views=[dict(w=1280, h=720, gaze=[640.0, 360.0])],
        K=4, active_sh=1, background=0, blur=False, to_chw=True, aaa=False),
    "stereo_fast_tex_hwc": dict(
        module="_C_stereo", n=8000, sh_degree=3, seed=14, views=[dict(w=520, h=560, gaze=[260.0, 280.0], eye=-0.0315),
                                                                 dict(w=520, h=560, gaze=[255.0, 283.0], eye=+0.0315)],
        K=8, active_sh=16, background=2, blur=False, to_chw=False, aaa=False),
}


def case_inputs(c: dict):
    """Deterministic inputs of a case: (Gaussians, [View], background array or None)."""
    g = scene.make_gaussians(c["n"], c["sh_degree"], seed=c["seed"])
    views = []
    for v in c["views"]:
        gl = (-(-v["w"] // 16), -(-v["h"] // 16))
        vis = scene.random_visibility(gl[0], gl[1], v["mask_p"], v["mask_seed"]) if "mask_p" in v else None
        view = scene.make_view(v["w"], v["h"], eye_offset=v.get("eye", 0.0), visible=vis)
        view.gaze_position = np.asarray(v["gaze"], np.float32)
        views.append(view)
    bg = None
    if c["background"] == 1:
        bg = scene.sh_background(c["seed"])
    elif c["background"] in (2, 3):
        bg = scene.texture_background(64, 32, seed=c["seed"], raw=c["background"] == 3)
    return g, views, bg


def _settings(view, c, bg, device):
    from foveatedhtgscudabackend_b200 import BackgroundModel, settings_from_view
    return settings_from_view(view, K=c["K"], active_sh_bases=c["active_sh"], background=BackgroundModel(c["background"]),
                              background_data=bg, device=device)


def reference_outputs(c: dict) -> dict:
    import torch

    from foveatedhtgscudabackend_b200 import gaussians_to_torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref  # noqa: E402

    g, views, bg = case_inputs(c)
    gt = gaussians_to_torch(g, "cuda")
    st = [_settings(v, c, bg, "cuda") for v in views]
    fast = c["module"] != "_C"
    out: dict = {}
    for i, s in enumerate(st):
        inter = ref.intermediates(gt, s, fast=fast, aaa=c["aaa"])
        for k, val in inter.items():
            out[f"v{i}_{k}"] = np.asarray(val)
    mod = ref.module(c["module"])
    args = (c["to_chw"], c["blur"], c["aaa"])
    if c["module"] == "_C_stereo":
        a, b = mod.render(*gt, *st[0].as_tuple(), *st[1].as_tuple(), *args)
        torch.cuda.synchronize()
        out["v0_image"] = a.cpu().numpy()
        out["v1_image"] = b.cpu().numpy()
    else:
        fn = mod.render if c["module"] == "_C" else mod.benchmark
        img = fn(*gt, *st[0].as_tuple(), *args)
        torch.cuda.synchronize()
        out["v0_image"] = img.cpu().numpy()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    for name in a.cases:
        res = reference_outputs(CASES[name])
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), **res)
        with open(os.path.join(a.out, f"{name}.json"), "w") as f:
            json.dump(CASES[name], f, indent=1, sort_keys=True)
        print(name, {k: v.shape for k, v in res.items() if hasattr(v, "shape")})
    return 0


if __name__ == "__main__":
    sys.exit(main())
