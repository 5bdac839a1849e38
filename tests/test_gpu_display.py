"""GPU parity of the kernels either side of the rendering path, through the C ABI.

* tile masks built on the device == the restatement (and the scene's host tables), bit-exact,
  and a frame rendered with them == the frame rendered with host-built masks;
* display packing == the restatement, bit-exact, including a full-size stereo frame;
* the two debug overlays == the reference's own `_C_visualization` output (golden images,
  bit-exact), == the restatement, and == the live reference module when it is built here.
"""
import os

import numpy as np
import pytest
import torch

import display_oracle as D
import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import scene
from golden.make_golden_visualization import GREY, ORACLE_ONLY_TILE_CASES, all_cases, case_inputs

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "visualization", "reference_overlays.npz")


def ours(name: str) -> np.ndarray:
    img, kind, a = case_inputs(name)
    t = torch.from_numpy(img).to(DEV)
    vis = F.FoveatedHTGSVisualizer()
    if kind == "gaze":
        out = vis.visualize_gaze(t, torch.from_numpy(a["gaze"]), torch.from_numpy(a["color"]), a["size"], a["vtype"],
                                 a["to_chw"])
    else:
        mask = torch.from_numpy(a["mask"].view(np.int32)).to(DEV).view(torch.uint32)
        out = vis.visualize_tile_boundaries(t, mask, torch.from_numpy(a["gaze"]), a["to_chw"])
    assert out is t  # drawn in place, like the reference
    torch.cuda.synchronize()
    return t.cpu().numpy()


def oracle(name: str) -> np.ndarray:
    img, kind, a = case_inputs(name)
    if kind == "gaze":
        return D.visualize_gaze(img, a["gaze"], a["color"], a["size"], a["vtype"], a["to_chw"])
    return D.visualize_tile_boundaries(img, a["mask"], a["gaze"], a["to_chw"])


@pytest.mark.parametrize("name", all_cases())
def test_overlays_bit_identical_to_reference_golden_and_oracle(name):
    golden = dict(np.load(FIXTURE))[name]
    out = ours(name)
    assert np.array_equal(out, golden), f"{name}: {int(np.sum(out != golden))} values differ from the reference"
    assert np.array_equal(out, oracle(name))


def test_overlay_with_no_visible_tile_draws_nothing():
    for name in ORACLE_ONLY_TILE_CASES:
        assert np.all(ours(name) == GREY)


def _live_reference():
    import ref
    if not os.path.exists(os.path.join(ref.REF_DIR, "FoveatedHTGSCudaBackend")):
        return None
    try:
        return ref.module("_C_visualization")
    except ImportError:
        return None


def test_overlays_match_live_reference_module():
    mod = _live_reference()
    if mod is None:
        pytest.skip("reference _C_visualization not built under oracle/_ref")
    for name in all_cases():
        img, kind, a = case_inputs(name)
        t = torch.from_numpy(img).to(DEV)
        if kind == "gaze":
            mod.visualize_gaze(t, torch.from_numpy(a["gaze"]), torch.from_numpy(a["color"]), a["vtype"], a["size"],
                               a["to_chw"])
        else:
            mask = torch.from_numpy(a["mask"].view(np.int32)).to(DEV).view(torch.uint32)
            mod.visualize_tile_boundaries(t, mask, torch.from_numpy(a["gaze"]), a["to_chw"])
        torch.cuda.synchronize()
        assert np.array_equal(t.cpu().numpy(), ours(name)), name


@pytest.mark.parametrize("w,h,vis", [(2064, 2208, None), (2064, 2208, "random"), (640, 480, "lens"), (1, 1, None),
                                     (513, 1, "random"), (16 * 32, 16 * 2, "random"), (1003, 757, "lens"),
                                     (8192, 8192, "random")])
def test_device_tile_masks_match_oracle(w, h, vis):
    gw, gh = -(-w // 16), -(-h // 16)
    visible = None
    if vis == "random":
        visible = scene.random_visibility(gw, gh, 0.6, w + h)
    elif vis == "lens":
        visible = scene.lens_visibility(gw, gh)
    vt = None if visible is None else torch.from_numpy(visible).to(DEV)
    words, sat, fov = F.build_tile_masks(w, h, vt, device=DEV)
    torch.cuda.synchronize()
    o_words, o_sat, o_fov = D.tile_masks(w, h, visible) if gw * gh <= 20000 else (
        *scene.visibility_tables(gw, gh, visible), scene.fovea_table())
    assert words.dtype == torch.uint32 and sat.dtype == torch.uint32
    assert np.array_equal(words.cpu().numpy(), o_words)
    assert np.array_equal(sat.cpu().numpy(), o_sat)
    assert np.array_equal(fov.cpu().numpy(), o_fov)


def test_frame_rendered_with_device_masks_equals_host_masks():
    g = scene.make_gaussians(20000, 3, seed=5)
    w, h = 640, 480
    visible = scene.random_visibility(40, 30, 0.8, 9)
    v = scene.make_view(w, h, visible=visible, gaze_ndc=(0.2, -0.1))
    gt = F.gaussians_to_torch(g)
    s_host = F.settings_from_view(v, K=8, active_sh_bases=16)
    words, sat, fov = F.build_tile_masks(w, h, torch.from_numpy(visible).to(DEV))
    s_dev = s_host._replace(visibility_mask=words, visibility_mask_area_table=sat, fovea_mask_area_table=fov)
    r = F.FoveatedHTGSRasterizer()
    a = r.benchmark(*gt, s_host, True, False, False)
    b = r.benchmark(*gt, s_dev, True, False, False)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


@pytest.mark.parametrize("n_views,to_chw,bgra", [(1, True, False), (2, False, True), (3, True, True)])
def test_pack_display_matches_oracle(n_views, to_chw, bgra):
    rng = np.random.default_rng(n_views)
    h, w = 37, 53
    imgs = [rng.uniform(-0.2, 1.2, (3, h, w) if to_chw else (h, w, 3)).astype(np.float32) for _ in range(n_views)]
    imgs[0].reshape(-1)[:6] = [np.nan, np.inf, -np.inf, 0.5, 1.0, 0.0]
    out = F.pack_display([torch.from_numpy(i).to(DEV) for i in imgs], to_chw=to_chw, bgra=bgra)
    torch.cuda.synchronize()
    assert out.shape == (h, n_views * w, 4) and out.dtype == torch.uint8
    assert np.array_equal(out.cpu().numpy(), D.pack_display(imgs, to_chw=to_chw, bgra=bgra))


def test_pack_display_full_size_stereo_frame():
    g = scene.make_gaussians(50000, 3, seed=3)
    left, right = scene.make_stereo_views(2064, 2208, seed=0)
    gt = F.gaussians_to_torch(g)
    st = [F.settings_from_view(v, K=8, active_sh_bases=16) for v in (left, right)]
    a, b = F.FoveatedHTGSRasterizer().render_stereo(*gt, st[0], st[1], True, False, False)
    out = F.pack_display([a, b], to_chw=True)
    torch.cuda.synchronize()
    expect = D.pack_display([a.cpu().numpy(), b.cpu().numpy()], to_chw=True)
    assert np.array_equal(out.cpu().numpy(), expect)
