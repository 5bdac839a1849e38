"""Generates tests/golden/visualization/reference_overlays.npz from the REFERENCE's overlays.

Runs on a machine with a B200 and the reference's `_C_visualization` module built by
`oracle/build_ref.sh` (under oracle/_ref/).  Every case below starts from a constant-grey
image (the grey marks pixels an overlay must leave alone), calls the reference's
`visualize_gaze` or `visualize_tile_boundaries` through its own pybind entry point, and stores
the resulting image.  Inputs are rebuilt from the case parameters by `case_inputs`.

    python tests/golden/make_golden_visualization.py --out tests/golden/visualization
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

GREY = 0.25

# gaze markers: (width, height, to_chw, gaze, color, size, type)
GAZE_CASES = {
    "gaze_circle_16": (320, 200, True, (160.0, 100.0), (1.0, 0.0, 0.0), 16, 0),
    "gaze_circle_15_hwc": (320, 200, False, (100.7, 60.2), (0.0, 1.0, 0.0), 15, 0),
    "gaze_square_7": (320, 200, True, (10.0, 190.5), (0.0, 0.0, 1.0), 7, 1),
    "gaze_cross_40_hwc": (320, 200, False, (300.0, 5.0), (1.0, 1.0, 0.0), 40, 2),
    "gaze_cross_9": (320, 200, True, (-50.0, 400.0), (0.5, 0.25, 1.0), 9, 2),
    "gaze_circle_1": (320, 200, True, (0.0, 0.0), (1.0, 1.0, 1.0), 1, 0),
    "gaze_type5_square_12": (320, 200, False, (319.0, 199.0), (0.1, 0.2, 0.3), 12, 5),
    "gaze_circle_33_ragged": (83, 45, True, (41.5, 22.5), (0.9, 0.1, 0.4), 33, 0),
}

# tile boundaries: (width, height, to_chw, gaze, visibility) with visibility one of
# "all", ("random", p, seed), ("lens",), ("single", tile), ("none",)
TILE_CASES = {
    "tiles_all_center": (1000, 760, True, (500.0, 380.0), ("all",)),
    "tiles_random_hwc": (1000, 760, False, (260.3, 611.9), ("random", 0.7, 3)),
    "tiles_lens_corner": (1000, 760, True, (990.0, 2.0), ("lens",)),
    "tiles_ragged_outside": (1003, 757, False, (-40.0, 900.0), ("random", 0.9, 4)),
    "tiles_small_view": (200, 136, True, (90.0, 70.0), ("all",)),
    "tiles_single_periphery": (1000, 760, True, (100.0, 100.0), ("single", 62 * 1 + 60)),
    "tiles_single_fovea": (1000, 760, True, (100.0, 100.0), ("single", 63 * 6 + 6)),
    "tiles_two_periphery": (1000, 760, False, (100.0, 100.0), ("tiles", [63 * 40 + 60, 63 * 47 + 62])),
}
# With no visible tile the reference launches a kernel over zero tiles (an invalid launch
# configuration the runtime rejects, leaving a pending error for the next launch): that case is
# checked against the restatement only.
ORACLE_ONLY_TILE_CASES = {
    "tiles_none": (1000, 760, True, (500.0, 380.0), ("none",)),
}


def _visible(w: int, h: int, spec) -> np.ndarray:
    gw, gh = -(-w // 16), -(-h // 16)
    kind = spec[0]
    if kind == "all":
        return np.ones((gh, gw), bool)
    if kind == "none":
        return np.zeros((gh, gw), bool)
    if kind == "random":
        return scene.random_visibility(gw, gh, spec[1], spec[2])
    if kind == "lens":
        return scene.lens_visibility(gw, gh)
    v = np.zeros(gw * gh, bool)
    v[[spec[1]] if kind == "single" else spec[1]] = True
    return v.reshape(gh, gw)


def case_inputs(name: str):
    """(image [grey], kind, args) of a case; args are what the overlay call takes besides the image."""
    if name in GAZE_CASES:
        w, h, chw, gaze, color, size, vtype = GAZE_CASES[name]
        img = np.full((3, h, w) if chw else (h, w, 3), GREY, np.float32)
        return img, "gaze", dict(gaze=np.asarray(gaze, np.float32), color=np.asarray(color, np.float32), size=size,
                                 vtype=vtype, to_chw=chw)
    w, h, chw, gaze, spec = {**TILE_CASES, **ORACLE_ONLY_TILE_CASES}[name]
    img = np.full((3, h, w) if chw else (h, w, 3), GREY, np.float32)
    words, _ = scene.visibility_tables(-(-w // 16), -(-h // 16), _visible(w, h, spec))
    return img, "tiles", dict(gaze=np.asarray(gaze, np.float32), mask=words, to_chw=chw)


def all_cases() -> list[str]:
    return list(GAZE_CASES) + list(TILE_CASES)


def run_reference(name: str) -> np.ndarray:
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref  # noqa: E402

    mod = ref.module("_C_visualization")
    img, kind, a = case_inputs(name)
    t = torch.from_numpy(img).cuda()
    if kind == "gaze":
        mod.visualize_gaze(t, torch.from_numpy(a["gaze"]), torch.from_numpy(a["color"]), a["vtype"], a["size"],
                           a["to_chw"])
    else:
        mask = torch.from_numpy(a["mask"].view(np.int32)).cuda().view(torch.uint32)
        mod.visualize_tile_boundaries(t, mask, torch.from_numpy(a["gaze"]), a["to_chw"])
    torch.cuda.synchronize()
    return t.cpu().numpy()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "visualization"))
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    res = {name: run_reference(name) for name in all_cases()}
    np.savez_compressed(os.path.join(a.out, "reference_overlays.npz"), **res)
    with open(os.path.join(a.out, "reference_overlays.json"), "w") as f:
        json.dump({"gaze": {k: list(map(str, v)) for k, v in GAZE_CASES.items()},
                   "tiles": {k: list(map(str, v)) for k, v in TILE_CASES.items()}}, f, indent=1)
    for name, img in res.items():
        print(name, img.shape, int(np.sum(np.any((img != GREY), axis=0 if img.shape[0] == 3 else 2))))
    return 0


if __name__ == "__main__":
    sys.exit(main())
