"""GPU tests of the ring and no-foveation modes (FHTGS_FOVEATION_RINGS / _NONE), through the
C ABI (Renderer).  The reference has neither mode, so the CUDA path is checked against the CPU
oracle's restatement of them: PSNR >= 50 dB against the oracle in FP32 with the same (IEEE or
fast) arithmetic family, >= 40 dB against FP64.  Where a mode renders pixels exactly as another
does (sample positions, full-resolution tiles) the test asks for bit equality.
"""
import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import _lib, scene
import oracle as O
from helpers import psnr

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def g():
    return scene.make_gaussians(40000, 3, seed=12)


@pytest.fixture(scope="module")
def gt(g):
    return F.gaussians_to_torch(g, DEV)


def render(gt, views, mode="reference", rings=(0.15, 0.4), fast=False, blur=False):
    r = F.Renderer(DEV)
    try:
        r.set_foveation(mode, *rings)
        st = [F.settings_from_view(v, K=8, active_sh_bases=16, device=DEV) for v in views]
        return [x.cpu().numpy() for x in r.render(*gt, st, fast_math=fast, blur_periphery=blur)]
    finally:
        r.close()


CASES = [
    ("rings", (0.15, 0.4), (480, 400), (0.0, 0.0)),
    ("rings", (0.15, 0.4), (333, 217), (0.7, -0.6)),
    ("rings", (0.3, 0.6), (640, 352), (-1.3, 1.2)),   # gaze clamped to the corner
    ("rings", (0.0, 0.0), (272, 208), (0.1, 0.1)),    # all 4x
    ("none", (0.0, 0.0), (333, 217), (0.2, -0.3)),
]


@pytest.mark.parametrize("mode,rings,size,gaze", CASES)
@pytest.mark.parametrize("fast", [False, True])
def test_modes_match_the_oracle(g, gt, mode, rings, size, gaze, fast):
    v = scene.make_view(*size, gaze_ndc=gaze)
    img = render(gt, [v], mode, rings, fast)[0]
    o32 = O.render(g, v, K=8, active_sh_bases=16, precision=32, foveation=mode, rings=rings)
    o64 = O.render(g, v, K=8, active_sh_bases=16, precision=64, foveation=mode, rings=rings)
    assert img.max() > 0.0
    assert psnr(img, o32) >= 50.0, f"{mode} {rings} {size}: {psnr(img, o32):.1f} dB vs oracle FP32"
    assert psnr(img, o64) >= 40.0, f"{mode} {rings} {size}: {psnr(img, o64):.1f} dB vs oracle FP64"


def test_rings_with_masks_match_the_oracle(g, gt):
    w, h = 400, 320
    vis = scene.lens_visibility(-(-w // 16), -(-h // 16))
    v = scene.make_view(w, h, gaze_ndc=(0.2, 0.1), visible=vis)
    img = render(gt, [v], "rings", (0.2, 0.5))[0]
    o32 = O.render(g, v, K=8, active_sh_bases=16, precision=32, foveation="rings", rings=(0.2, 0.5))
    assert psnr(img, o32) >= 50.0


def test_large_rings_equal_no_foveation_bit_for_bit(gt):
    v = scene.make_view(333, 217, gaze_ndc=(0.3, 0.2))
    none = render(gt, [v], "none")[0]
    rings = render(gt, [v], "rings", (3.0, 3.0))[0]
    assert np.array_equal(none, rings)


def test_sample_positions_equal_full_resolution_bit_for_bit(gt):
    v = scene.make_view(480, 400, gaze_ndc=(0.0, 0.0))
    none = render(gt, [v], "none")[0]
    quarter = render(gt, [v], "rings", (0.0, 0.0))[0]
    half = render(gt, [v], "rings", (0.0, 3.0))[0]
    assert np.array_equal(quarter[:, ::4, ::4], none[:, ::4, ::4])
    assert np.array_equal(half[:, ::2, ::2], none[:, ::2, ::2])


def test_no_foveation_equals_reference_on_fovea_tiles(gt):
    v = scene.make_view(480, 400, gaze_ndc=(0.1, -0.1))
    ref = render(gt, [v], "reference")[0]
    none = render(gt, [v], "none")[0]
    geo = O.geometry(v)
    gx, gy = geo["gaze_tile_x"], geo["gaze_tile_y"]
    mask = np.zeros((v.height, v.width), bool)
    for ty in range(geo["grid_large_h"]):
        for tx in range(geo["grid_large_w"]):
            d2 = (np.float32(tx) + np.float32(0.5) - np.float32(gx)) ** 2 + (np.float32(ty) + np.float32(0.5) - np.float32(gy)) ** 2
            if d2 < 225:
                mask[ty * 16:ty * 16 + 16, tx * 16:tx * 16 + 16] = True
    assert mask.any()
    assert np.array_equal(ref[:, mask], none[:, mask])


def test_ring_frames_of_many_views_equal_views_alone(gt):
    views = scene.make_batched_views(5, seed=4, radius=(3.0, 6.0), resolutions=((320, 240), (272, 400), (96, 64)))
    together = render(gt, views, "rings", (0.2, 0.45))
    for i, v in enumerate(views):
        alone = render(gt, [v], "rings", (0.2, 0.45))[0]
        assert np.array_equal(alone, together[i]), f"view {i}"


def test_invalid_ring_settings_are_rejected(gt):
    v = scene.make_view(160, 120)
    with pytest.raises(_lib.FhtgsError):
        render(gt, [v], "rings", (0.15, 0.4), blur=True)
    with pytest.raises(_lib.FhtgsError):
        render(gt, [v], "rings", (0.5, 0.4))
    with pytest.raises(ValueError):
        render(gt, [v], "spiral")


def test_per_view_foveation_in_one_frame_equals_views_alone(gt):
    """Views of one frame may carry their own foveation; each equals the view rendered alone
    with that foveation for the whole frame."""
    views = scene.make_batched_views(4, seed=8, radius=(3.0, 6.0), resolutions=((320, 240), (272, 400)))
    modes = ["none", ("rings", 0.15, 100.0), ("rings", 0.15, 0.4), "reference"]
    r = F.Renderer(DEV)
    try:
        st = [F.settings_from_view(v, K=8, active_sh_bases=16, device=DEV) for v in views]
        together = [x.cpu().numpy() for x in r.render(*gt, st, fast_math=False, view_foveation=modes)]
    finally:
        r.close()
    for i, (v, m) in enumerate(zip(views, modes)):
        mode, radii = (m, (0.15, 0.4)) if isinstance(m, str) else (m[0], m[1:])
        alone = render(gt, [v], mode, radii)[0]
        assert np.array_equal(alone, together[i]), f"view {i} ({m})"


def test_captured_graph_with_per_view_foveation_equals_eager(gt):
    """A frame graph captured with per-view foveation replays the eager frame bit for bit, and
    the frame information afterwards reports each view in its own layout."""
    views = scene.make_batched_views(3, seed=9, radius=(3.0, 6.0), resolutions=((320, 240), (272, 400)))
    modes = [("rings", 0.15, 0.4), "reference", "none"]
    r = F.Renderer(DEV)
    try:
        st = [F.settings_from_view(v, K=8, active_sh_bases=16, device=DEV) for v in views]
        eager = [x.clone() for x in r.render(*gt, st, view_foveation=modes)]
        graph = r.capture(*gt, st, capacity_headroom=1.5, view_foveation=modes)
        try:
            replay = graph.launch(sync=True)
            for a, b in zip(eager, replay):
                assert torch.equal(a, b)
            info = [r.frame_info(i) for i in range(3)]
            assert all(not i["overflow"] for i in info)
        finally:
            graph.close()
    finally:
        r.close()
