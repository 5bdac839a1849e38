"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

* golden fixtures (tests/golden, produced by the reference itself): integer intermediates
  bit-exact, images within max-abs 2e-3 and PSNR >= 50 dB;
* the live reference (oracle/_ref, when present on the machine): same bars on fresh seeds and at
  the full headline size;
* the CPU oracle: stage-wise (instances from our per-primitive outputs must match exactly; the
  FP32 blend of our intermediates must match our image) and end-to-end against FP64.
"""
import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import scene
import oracle as O
import ref as REF
from golden.make_golden import CASES, case_inputs
from helpers import (REF_MAX_ABS, REF_PSNR_DB, assert_instances_equal, assert_tiles_equal, golden_cases, load_golden,
                     max_abs, psnr, view_data)

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not REF.available(), reason="reference build (oracle/_ref) not present")


@pytest.fixture(scope="module")
def renderer():
    r = F.Renderer("cuda:0")
    yield r
    r.close()


def settings_for(c, views, bg):
    return [F.settings_from_view(v, K=c["K"], active_sh_bases=c["active_sh"],
                                 background=F.BackgroundModel(c["background"]), background_data=bg) for v in views]


def render_case(renderer, c, *, fast=None):
    g, views, bg = case_inputs(c)
    gt = F.gaussians_to_torch(g)
    st = settings_for(c, views, bg)
    fast = (c["module"] != "_C") if fast is None else fast
    imgs = renderer.render(*gt, st, to_chw=c["to_chw"], blur_periphery=c["blur"], aaa_mode=c["aaa"], fast_math=fast)
    torch.cuda.synchronize()
    inter = [renderer.intermediates(i) for i in range(len(views))]
    return g, views, bg, gt, st, [i.cpu().numpy() for i in imgs], inter


def assert_primitives_equal(mine, ref, what=""):
    nt_m, nt_r = np.asarray(mine["n_touched"]), np.asarray(ref["n_touched"])
    assert np.array_equal(nt_m, nt_r), f"{what}: n_touched differs for {np.count_nonzero(nt_m != nt_r)} primitives"
    live = nt_r > 0
    sb_m, sb_r = np.asarray(mine["screen_bounds"])[live], np.asarray(ref["screen_bounds"])[live]
    assert np.array_equal(sb_m, sb_r), f"{what}: screen bounds differ"
    for k in ("vpmt", "rgba"):
        a, b = np.asarray(mine[k])[live], np.asarray(ref[k])[live]
        diff = a.view(np.uint32) != b.view(np.uint32)
        assert not diff.any(), (f"{what}: {k} not bit-identical for {diff.any(1).sum()} of {live.sum()} primitives, "
                                f"max abs diff {np.abs(a - b).max():.3g}")


def assert_image_close(mine, ref, what=""):
    ma, p = max_abs(mine, ref), psnr(mine, ref)
    assert ma <= REF_MAX_ABS and p >= REF_PSNR_DB, f"{what}: max-abs {ma:.3g}, PSNR {p:.1f} dB"


# ---------------------------------------------------------------------------------------------
# golden fixtures (reference outputs)
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", golden_cases())
def test_intermediates_bit_exact_vs_golden(renderer, name):
    case, data = load_golden(name)
    _, views, _, _, _, _, inter = render_case(renderer, case)
    for i in range(len(views)):
        ref = view_data(data, i)
        what = f"{name}/view{i}"
        assert_primitives_equal(inter[i], ref, what)
        assert_tiles_equal(inter[i], ref, what)
        assert_instances_equal(inter[i], ref, int(ref["end_bit"]), what)


@pytest.mark.parametrize("name", golden_cases())
def test_images_bit_identical_vs_golden(renderer, name):
    """The blend keeps the reference's per-pixel arithmetic and order: images match bit for bit."""
    case, data = load_golden(name)
    g, views, bg = case_inputs(case)
    imgs = renderer.render(*F.gaussians_to_torch(g), settings_for(case, views, bg), to_chw=case["to_chw"],
                           blur_periphery=case["blur"], aaa_mode=case["aaa"], fast_math=case["module"] != "_C")
    for i, im in enumerate(imgs):
        a, b = im.cpu().numpy(), data[f"v{i}_image"]
        assert np.array_equal(a, b), f"{name}/view{i}: {np.count_nonzero(a != b)} values differ, max {max_abs(a, b):.3g}"


@pytest.mark.parametrize("name", golden_cases())
def test_dropin_images_vs_golden(name):
    case, data = load_golden(name)
    g, views, bg = case_inputs(case)
    gt = F.gaussians_to_torch(g)
    st = settings_for(case, views, bg)
    args = (case["to_chw"], case["blur"], case["aaa"])
    if case["module"] == "_C_stereo":
        imgs = F._C_stereo.render(*gt, *st[0].as_tuple(), *st[1].as_tuple(), *args)
    elif case["module"] == "_C":
        imgs = (F._C.render(*gt, *st[0].as_tuple(), *args),)
    else:
        imgs = (F._C_benchmarking.benchmark(*gt, *st[0].as_tuple(), *args),)
    for i, im in enumerate(imgs):
        assert_image_close(im.cpu().numpy(), data[f"v{i}_image"], f"{name}/view{i}")


# ---------------------------------------------------------------------------------------------
# live reference on fresh inputs
# ---------------------------------------------------------------------------------------------
LIVE = [
    dict(module="_C_benchmarking", n=40000, sh_degree=3, seed=101, views=[dict(w=1280, h=720, gaze=[300.0, 200.0],
         mask_p=0.9, mask_seed=3)], K=8, active_sh=16, background=0, blur=False, to_chw=True, aaa=False),
    dict(module="_C", n=30000, sh_degree=2, seed=102, views=[dict(w=960, h=540, gaze=[900.0, 30.0])], K=2,
         active_sh=9, background=1, blur=True, to_chw=False, aaa=True),
    dict(module="_C_stereo", n=30000, sh_degree=3, seed=103, views=[dict(w=1032, h=1104, gaze=[500.0, 560.0], eye=-0.0315),
         dict(w=900, h=1000, gaze=[470.0, 520.0], eye=0.0315)], K=32, active_sh=16, background=2, blur=False,
         to_chw=True, aaa=False),
    # the plain single-view config (100k SH0 Gaussians, 1280x720, K = 4, centred gaze): an
    # instance count for which the reference's own module skips its sort, so its images are
    # checked through the oracle while its kernels (through the harness) are compared exactly
    dict(module="_C_benchmarking", n=100000, sh_degree=0, seed=0, views=[dict(w=1280, h=720, gaze=[640.0, 360.0])],
         K=4, active_sh=1, background=0, blur=False, to_chw=True, aaa=False),
]


@needs_ref
@pytest.mark.parametrize("ci", range(len(LIVE)))
def test_live_reference_intermediates_and_images(renderer, ci):
    c = LIVE[ci]
    g, views, bg, gt, st, imgs, inter = render_case(renderer, c)
    fast = c["module"] != "_C"
    for i in range(len(views)):
        ref = REF.intermediates(gt, st[i], fast=fast, aaa=c["aaa"])
        what = f"live{ci}/view{i}"
        assert_primitives_equal(inter[i], ref, what)
        assert_tiles_equal(inter[i], ref, what)
        assert_instances_equal(inter[i], ref, ref["end_bit"], what)
    mod = REF.module(c["module"])
    args = (c["to_chw"], c["blur"], c["aaa"])

    def ref_images():
        if c["module"] == "_C_stereo":
            out = mod.render(*gt, *st[0].as_tuple(), *st[1].as_tuple(), *args)
        else:
            out = ((mod.render if c["module"] == "_C" else mod.benchmark)(*gt, *st[0].as_tuple(), *args),)
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in out]

    first, second = ref_images(), ref_images()
    for i in range(len(views)):
        if np.array_equal(first[i], second[i]):
            assert_image_close(imgs[i], first[i], f"live{ci}/view{i}")
        else:
            # The reference does not reproduce itself on this input (observed for the left eye
            # of _C_stereo: fovea tiles left unwritten); the oracle is the judge here.
            kw = dict(K=c["K"], active_sh_bases=c["active_sh"], to_chw=c["to_chw"], blur=c["blur"], aaa=c["aaa"],
                      background=bg, background_type=c["background"], precision=32)
            p = psnr(imgs[i], O.render(g, views[i], **kw))
            assert p >= 80.0, f"live{ci}/view{i}: reference not reproducible; PSNR vs oracle {p:.1f} dB"


@needs_ref
def test_headline_size_stereo_vs_reference(renderer):
    """Stereo 2 x 2064x2208, 1M Gaussians SH3, K=8 (the benchmark workload), fast-math."""
    g = scene.make_gaussians(1_000_000, 3, seed=0)
    L, R = scene.make_stereo_views(2064, 2208, seed=0)
    gt = F.gaussians_to_torch(g)
    st = [F.settings_from_view(v, K=8, active_sh_bases=16) for v in (L, R)]
    mine = F._C_stereo.render(*gt, *st[0].as_tuple(), *st[1].as_tuple(), True, False, False)
    refm = REF.module("_C_stereo").render(*gt, *st[0].as_tuple(), *st[1].as_tuple(), True, False, False)
    for i in range(2):
        assert_image_close(mine[i].cpu().numpy(), refm[i].cpu().numpy(), f"headline/view{i}")
    renderer.render(*gt, st, to_chw=True, fast_math=True)
    for i in range(2):
        ref = REF.intermediates(gt, st[i], fast=True)
        m = renderer.intermediates(i)
        assert_primitives_equal(m, ref, f"headline/view{i}")
        assert_tiles_equal(m, ref, f"headline/view{i}")
        assert_instances_equal(m, ref, ref["end_bit"], f"headline/view{i}")


# ---------------------------------------------------------------------------------------------
# oracle (CPU restatement)
# ---------------------------------------------------------------------------------------------
ORACLE_CASES = [
    dict(module="_C", n=6000, sh_degree=3, seed=201, views=[dict(w=640, h=480, gaze=[100.0, 80.0], mask_p=0.8,
         mask_seed=9)], K=8, active_sh=16, background=1, blur=False, to_chw=True, aaa=False),
    dict(module="_C", n=6000, sh_degree=3, seed=202, views=[dict(w=640, h=480, gaze=[560.0, 400.0])], K=4,
         active_sh=16, background=3, blur=True, to_chw=False, aaa=True),
    dict(module="_C_benchmarking", n=6000, sh_degree=1, seed=203, views=[dict(w=500, h=300, gaze=[10.0, 10.0])],
         K=16, active_sh=4, background=2, blur=True, to_chw=True, aaa=False),
]


@pytest.mark.parametrize("ci", range(len(ORACLE_CASES)))
def test_stagewise_vs_oracle(renderer, ci):
    c = ORACLE_CASES[ci]
    g, views, bg, gt, st, imgs, inter = render_case(renderer, c)
    v, m = views[0], inter[0]
    # instance creation + stable sort + ranges from OUR per-primitive outputs: exact
    oi = O.instances(v, m["n_touched"], m["screen_bounds"])
    assert_instances_equal(m, oi, O.geometry(v)["end_bit"], "oracle instances")
    assert_tiles_equal(m, O.classify(v), "oracle tiles")
    # blend + compose of OUR intermediates in FP32 on the host: matches our image
    kw = dict(K=c["K"], active_sh_bases=c["active_sh"], to_chw=c["to_chw"], blur=c["blur"], aaa=c["aaa"],
              background=bg, background_type=c["background"], precision=32)
    im32 = O.blend_compose(v, g.n, m["vpmt"], m["rgba"], m["tile_index_map_partitioned"], m["partition_ranges"],
                           m["values"], m["instance_ranges"], **kw)
    assert psnr(imgs[0], im32) >= REF_PSNR_DB, f"PSNR vs FP32 oracle blend {psnr(imgs[0], im32):.1f} dB"
    # end to end against the FP64 oracle
    kw["precision"] = 64
    im64 = O.render(g, v, **kw)
    assert psnr(imgs[0], im64) >= 40.0, f"PSNR vs FP64 oracle {psnr(imgs[0], im64):.1f} dB"


# ---------------------------------------------------------------------------------------------
# edge cases
# ---------------------------------------------------------------------------------------------
def _oracle_image(g, v, **kw):
    return O.render(g, v, precision=32, **kw)


def test_zero_gaussians_background_only(renderer):
    g = scene.make_gaussians(0, 3)
    v = scene.make_view(320, 240)
    bg = scene.sh_background(1)
    st = [F.settings_from_view(v, K=8, active_sh_bases=16, background=F.BackgroundModel.SH, background_data=bg)]
    img = renderer.render(*F.gaussians_to_torch(g), st, fast_math=False)[0].cpu().numpy()
    ref = _oracle_image(g, v, K=8, background=bg, background_type=1)
    assert psnr(img, ref) >= REF_PSNR_DB
    assert renderer.frame_info(0)["n_instances"] == 0


@pytest.mark.parametrize("which", ["all_masked", "one_tile", "random"])
def test_masks(renderer, which):
    g = scene.make_gaussians(5000, 3, seed=7)
    gw, gh = 40, 30
    if which == "all_masked":
        vis = np.zeros((gh, gw), bool)
    elif which == "one_tile":
        vis = np.zeros((gh, gw), bool)
        vis[29, 39] = True
    else:
        vis = scene.random_visibility(gw, gh, 0.5, 3)
    v = scene.make_view(640, 480, gaze_ndc=(-1.0, -1.0), visible=vis)
    st = [F.settings_from_view(v, K=8, active_sh_bases=16)]
    img = renderer.render(*F.gaussians_to_torch(g), st, fast_math=False)[0].cpu().numpy()
    ref = _oracle_image(g, v, K=8)
    assert psnr(img, ref) >= REF_PSNR_DB
    if which != "random":
        assert not img.any()


@pytest.mark.parametrize("w,h", [(1, 1), (17, 9), (33, 700), (2064, 8)])
def test_odd_image_sizes(renderer, w, h):
    g = scene.make_gaussians(3000, 1, seed=w)
    v = scene.make_view(w, h, gaze_ndc=(0.5, -0.5))
    st = [F.settings_from_view(v, K=4, active_sh_bases=4)]
    img = renderer.render(*F.gaussians_to_torch(g), st, fast_math=False)[0].cpu().numpy()
    assert psnr(img, _oracle_image(g, v, K=4, active_sh_bases=4)) >= REF_PSNR_DB


def test_large_footprints_use_cooperative_emission(renderer):
    g = scene.make_gaussians(3000, 0, seed=5)
    g.scales[:50] = 0.6  # footprints of hundreds of tiles
    v = scene.make_view(1280, 720, gaze_ndc=(0.1, 0.1))
    st = [F.settings_from_view(v, K=8, active_sh_bases=1)]
    gt = F.gaussians_to_torch(g)
    img = renderer.render(*gt, st, fast_math=False)[0].cpu().numpy()
    m = renderer.intermediates(0)
    oi = O.instances(v, m["n_touched"], m["screen_bounds"])
    assert_instances_equal(m, oi, O.geometry(v)["end_bit"], "large footprints")
    assert psnr(img, _oracle_image(g, v, K=8, active_sh_bases=1)) >= REF_PSNR_DB


def test_wide_grid_uses_32bit_keys_and_three_sort_passes(renderer):
    """4400 x 4200: 72,325 large tiles, so stored keys are 32-bit with 17 significant bits
    (three onesweep passes) and the reference's keys 19-bit; instances exact vs the oracle."""
    g = scene.make_gaussians(20000, 0, seed=9)
    v = scene.make_view(4400, 4200, position=(0.0, 0.0, -4.5), gaze_ndc=(0.2, -0.1))
    st = [F.settings_from_view(v, K=8, active_sh_bases=1)]
    img = renderer.render(*F.gaussians_to_torch(g), st, fast_math=False)[0].cpu().numpy()
    m = renderer.intermediates(0)
    geo = O.geometry(v)
    assert geo["grid_large_w"] * geo["grid_large_h"] > 65536 and geo["end_bit"] > 16
    oi = O.instances(v, m["n_touched"], m["screen_bounds"])
    assert_instances_equal(m, oi, geo["end_bit"], "32-bit keys")
    assert psnr(img, _oracle_image(g, v, K=8, active_sh_bases=1)) >= REF_PSNR_DB


def test_capacity_overflow_grows_and_rerenders():
    r = F.Renderer("cuda:0")
    try:
        g = scene.make_gaussians(20000, 0, seed=8)
        v = scene.make_view(640, 480)
        r.reserve(g.n, 1, 640, 480, instances_per_view=4096)
        st = [F.settings_from_view(v, K=8, active_sh_bases=1)]
        img = r.render(*F.gaussians_to_torch(g), st, fast_math=False)[0].cpu().numpy()
        info = r.frame_info(0)
        assert info["n_instances"] > 4096 and not info["overflow"]
        assert psnr(img, _oracle_image(g, v, K=8, active_sh_bases=1)) >= REF_PSNR_DB
    finally:
        r.close()


@pytest.mark.parametrize("K", [1, 2, 4, 8, 16, 32])
def test_k_dispatch_vs_oracle(renderer, K):
    g = scene.make_gaussians(4000, 2, seed=40 + K)
    v = scene.make_view(400, 300, gaze_ndc=(0.7, 0.7))
    st = [F.settings_from_view(v, K=K, active_sh_bases=9)]
    img = renderer.render(*F.gaussians_to_torch(g), st, fast_math=False)[0].cpu().numpy()
    assert psnr(img, _oracle_image(g, v, K=K, active_sh_bases=9)) >= REF_PSNR_DB


def test_many_views_one_frame_equal_single_view_frames(renderer):
    g = scene.make_gaussians(8000, 3, seed=77)
    gt = F.gaussians_to_torch(g)
    rng = np.random.default_rng(0)
    views = []
    for i in range(5):
        w, h = [(320, 240), (640, 480), (500, 700)][i % 3]
        ang = rng.uniform(0, 2 * np.pi)
        pos = (6 * np.sin(ang), rng.uniform(-1, 1), -6 * np.cos(ang))
        views.append(scene.make_view(w, h, position=pos, gaze_ndc=tuple(rng.normal(0, 0.3, 2))))
    st = [F.settings_from_view(v, K=8, active_sh_bases=16) for v in views]
    together = [i.cpu().numpy() for i in renderer.render(*gt, st)]
    for i, s in enumerate(st):
        alone = renderer.render(*gt, [s])[0].cpu().numpy()
        assert np.array_equal(alone, together[i])


def test_invalid_inputs_raise(renderer):
    g = scene.make_gaussians(100, 0, seed=1)
    v = scene.make_view(64, 64)
    st = [F.settings_from_view(v, K=8, active_sh_bases=16)]  # SH degree 0 data, 16 bases requested
    with pytest.raises(F.FhtgsError):
        renderer.render(*F.gaussians_to_torch(g), st)
