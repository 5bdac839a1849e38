"""GPU tests of the split blend (a tolerance mode, off by default) through the C ABI.

With the mode on, a full-resolution tile whose list is long is blended as contiguous segments
on different blocks and merged by the last of them (fhtgs_context_set_blend_split).  The merge
replays every K-buffer insertion and eviction of the serial walk (reference blend_cu,
inference.cuh:188-240), so only the tail's float summation order changes.  Checked here:
- images within the reference tolerance (max-abs 2e-3, >= 50 dB) of the bit-identical path
  (itself bit-identical to the reference's images), with the differing pixels counted, and
  against the CPU FP64 oracle;
- run-to-run determinism, and a captured frame graph equal to the eager frame;
- a record overflow: every split tile is blended whole, serially, and the image is then
  bit-identical to the default path;
- the default (mode off) is untouched.
"""
import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
import oracle as O
from foveatedhtgscudabackend_b200 import _lib, scene
from helpers import REF_MAX_ABS, REF_PSNR_DB, max_abs, psnr

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def stereo():
    g = scene.make_gaussians(200_000, 3, seed=41)
    left, right = scene.make_stereo_views(800, 720, seed=5)
    return g, F.gaussians_to_torch(g, DEV), (left, right)


def render(gt, views, K=8, share=0.0, records=0, stats=False, **kw):
    st = [F.settings_from_view(v, K=K, active_sh_bases=16) for v in views]
    r = F.Renderer(DEV)
    try:
        r.set_blend_split(share, records)
        imgs = [x.clone() for x in r.render(*gt, st, **kw)]
        return (imgs, r.blend_split_stats()) if stats else imgs
    finally:
        r.close()


def compare(exact, split):
    a = torch.stack(exact).cpu().numpy()
    b = torch.stack(split).cpu().numpy()
    diff = np.abs(a.astype(np.float64) - b)
    return psnr(a, b), max_abs(a, b), int(np.count_nonzero(diff.max(axis=1))), a[0].shape[-1] * a[0].shape[-2] * len(a)


@pytest.mark.parametrize("K", [1, 8, 32])
@pytest.mark.parametrize("fast_math", [True, False])
def test_split_within_tolerance_of_exact_path(stereo, K, fast_math):
    _, gt, views = stereo
    exact = render(gt, views, K=K, fast_math=fast_math)
    split, stats = render(gt, views, K=K, share=0.1, stats=True, fast_math=fast_math)
    assert stats["split_tiles"] > 0 and stats["segments"] > stats["split_tiles"]
    assert stats["whole_fallbacks"] == 0
    p, m, n_diff, n_px = compare(exact, split)
    print(f"K={K} fast={fast_math}: {stats}, PSNR {p:.1f} dB, max-abs {m:.2e}, {n_diff}/{n_px} pixels differ")
    assert m <= REF_MAX_ABS and p >= REF_PSNR_DB
    assert m <= 1e-4  # rounding of the tail sums only


def test_split_is_deterministic_and_default_untouched(stereo):
    _, gt, views = stereo
    a = render(gt, views, share=0.1)
    b = render(gt, views, share=0.1)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    exact = render(gt, views)
    off = render(gt, views, share=0.0)
    for x, y in zip(exact, off):
        assert torch.equal(x, y)


def test_record_overflow_blends_split_tiles_whole(stereo):
    _, gt, views = stereo
    exact = render(gt, views)
    split, stats = render(gt, views, share=0.1, records=1, stats=True)
    assert stats["split_tiles"] > 0
    assert stats["whole_fallbacks"] == stats["split_tiles"]
    for x, y in zip(exact, split):
        assert torch.equal(x, y)


@pytest.mark.parametrize("case", ["blur", "sh_background", "rings", "aaa"])
def test_split_other_paths(stereo, case):
    _, gt, views = stereo
    kw, st_kw = {}, {}
    if case == "blur":
        kw = dict(blur_periphery=True)
    elif case == "aaa":
        kw = dict(aaa_mode=True)
    elif case == "rings":
        kw = dict(view_foveation=[("rings", 0.3, 0.6)] * 2)
    elif case == "sh_background":
        st_kw = dict(background=F.BackgroundModel.SH, background_data=scene.sh_background(3))
    out = []
    for share in (0.0, 0.1):
        st = [F.settings_from_view(v, K=8, active_sh_bases=16, **st_kw) for v in views]
        r = F.Renderer(DEV)
        r.set_blend_split(share, 0)
        out.append([x.clone() for x in r.render(*gt, st, **kw)])
        stats = r.blend_split_stats()
        r.close()
    assert stats["split_tiles"] > 0 and stats["whole_fallbacks"] == 0
    p, m, n_diff, n_px = compare(*out)
    print(f"{case}: PSNR {p:.1f} dB, max-abs {m:.2e}, {n_diff}/{n_px} pixels differ")
    assert m <= REF_MAX_ABS and p >= REF_PSNR_DB


def test_split_graph_equals_eager(stereo):
    _, gt, views = stereo
    st = [F.settings_from_view(v, K=8, active_sh_bases=16) for v in views]
    r = F.Renderer(DEV)
    r.set_blend_split(0.1, 0)
    eager = [x.clone() for x in r.render(*gt, st)]
    graph = r.capture(*gt, st, capacity_headroom=2.0)
    imgs = graph.launch(sync=True)
    for a, b in zip(eager, imgs):
        assert torch.equal(a, b)
    graph.close()
    r.close()


def test_split_accuracy_vs_fp64_oracle():
    g = scene.make_gaussians(40000, 3, seed=32)
    v = scene.make_view(480, 400, gaze_ndc=(0.1, -0.1))
    gt = F.gaussians_to_torch(g, DEV)
    exact = render(gt, [v], fast_math=False)[0].cpu().numpy()
    split, stats = render(gt, [v], share=0.05, stats=True, fast_math=False)
    split = split[0].cpu().numpy()
    assert stats["split_tiles"] > 0 and stats["whole_fallbacks"] == 0
    ref64 = O.render(g, v, K=8, active_sh_bases=16, precision=64)
    pe, ps = psnr(exact, ref64), psnr(split, ref64)
    print(f"vs FP64 oracle: exact {pe:.2f} dB, split {ps:.2f} dB (max-abs {max_abs(split, ref64):.2e})")
    assert ps >= REF_PSNR_DB and abs(ps - pe) < 0.5


def test_split_arguments_are_checked():
    r = F.Renderer(DEV)
    for share, rec in ((0.01, 0), (9.0, 0), (-1.0, 0), (0.5, -1), (0.5, 257)):
        with pytest.raises(_lib.FhtgsError):
            r.set_blend_split(share, rec)
    for log_bytes in (1000, -1, 65 << 30):
        with pytest.raises(_lib.FhtgsError):
            r.set_blend_split(0.5, 0, exact=True, log_bytes=log_bytes)
    r.set_blend_split(0.0, 0)
    r.close()


def test_server_with_split_blend(stereo):
    """The request server's frames with the split blend on (config blend_split_permille): every
    request within rounding of the bit-identical images, alone or fused with others."""
    from foveatedhtgscudabackend_b200.serving import Server
    _, gt, (left, right) = stereo
    exact = render(gt, (left, right))
    with Server(DEV, max_in_flight=2, max_batch_requests=4, blend_split=0.1) as srv:
        sid = srv.add_scene(*gt, K=8, active_sh_bases=16)
        srv.pause()
        for k in range(4):
            srv.submit(sid, [left, right], tag=k)
        srv.resume()
        got = {}
        while len(got) < 4:
            cs = srv.poll(wait_ms=5000)
            assert cs, "server made no progress"
            for c in cs:
                assert c.ok, c.message
                got[c.tag] = [x.clone() for x in c.images]
                srv.release(c.ticket)
    for k in range(4):
        p, m, n_diff, n_px = compare(exact, got[k])
        assert m <= 1e-4 and p >= REF_PSNR_DB, f"request {k}: max-abs {m}"
    with pytest.raises(_lib.FhtgsError):
        Server(DEV, blend_split=0.01)


def test_split_in_a_batch_of_mixed_views():
    """Eight cameras of mixed resolution and gaze in one frame, with per-view foveation: the
    split blend within rounding of the bit-identical batch."""
    g = scene.make_gaussians(150_000, 3, seed=43)
    views = scene.make_batched_views(8, seed=7, radius=(3.0, 6.0),
                                     resolutions=((320, 240), (640, 480), (272, 400), (800, 720)))
    gt = F.gaussians_to_torch(g, DEV)
    vf = ["none", ("rings", 0.15, 0.4), None, "none", ("rings", 0.3, 0.6), None, "none", None]
    out = []
    for share in (0.0, 0.1):
        st = [F.settings_from_view(v, K=8, active_sh_bases=16) for v in views]
        r = F.Renderer(DEV)
        r.set_blend_split(share, 0)
        out.append([x.clone() for x in r.render(*gt, st, view_foveation=vf)])
        stats = r.blend_split_stats()
        r.close()
    assert stats["split_tiles"] > 0 and stats["whole_fallbacks"] == 0
    for i, (a, b) in enumerate(zip(*out)):
        m = max_abs(a.cpu().numpy(), b.cpu().numpy())
        assert m <= 1e-4, f"view {i}: max-abs {m}"


# ---- the exact split: fragment logs replayed in list order, images bit-identical ----

def render_exact(gt, views, K=8, share=0.1, log_bytes=0, view_foveation=None, st_kw=None, **kw):
    st = [F.settings_from_view(v, K=K, active_sh_bases=16, **(st_kw or {})) for v in views]
    r = F.Renderer(DEV)
    try:
        r.set_blend_split(share, 0, exact=True, log_bytes=log_bytes)
        imgs = [x.clone() for x in r.render(*gt, st, view_foveation=view_foveation, **kw)]
        return imgs, r.blend_split_stats()
    finally:
        r.close()


@pytest.mark.parametrize("K", [1, 8, 32])
@pytest.mark.parametrize("fast_math", [True, False])
def test_exact_split_is_bit_identical(stereo, K, fast_math):
    _, gt, views = stereo
    exact = render(gt, views, K=K, fast_math=fast_math)
    split, stats = render_exact(gt, views, K=K, fast_math=fast_math)
    assert stats["split_tiles"] > 0 and stats["segments"] > stats["split_tiles"]
    for a, b in zip(exact, split):
        assert torch.equal(a, b), f"K={K}: {int((a != b).sum())} values differ, max {float((a - b).abs().max()):.3g}"


@pytest.mark.parametrize("case", ["blur", "sh_background", "rings", "aaa"])
def test_exact_split_other_paths(stereo, case):
    _, gt, views = stereo
    kw, st_kw, vf = {}, {}, None
    if case == "blur":
        kw = dict(blur_periphery=True)
    elif case == "aaa":
        kw = dict(aaa_mode=True)
    elif case == "rings":
        vf = [("rings", 0.3, 0.6)] * 2
    elif case == "sh_background":
        st_kw = dict(background=F.BackgroundModel.SH, background_data=scene.sh_background(3))
    st = [F.settings_from_view(v, K=8, active_sh_bases=16, **st_kw) for v in views]
    r = F.Renderer(DEV)
    exact = [x.clone() for x in r.render(*gt, st, view_foveation=vf, **kw)]
    r.close()
    split, stats = render_exact(gt, views, view_foveation=vf, st_kw=st_kw, **kw)
    assert stats["split_tiles"] > 0
    for a, b in zip(exact, split):
        assert torch.equal(a, b)


def test_exact_split_small_log_pool_leaves_tiles_whole(stereo):
    _, gt, views = stereo
    exact = render(gt, views)
    big, s_big = render_exact(gt, views)
    small, s_small = render_exact(gt, views, log_bytes=1 << 20)
    assert s_small["split_tiles"] < s_big["split_tiles"]
    for a, b, c in zip(exact, big, small):
        assert torch.equal(a, b) and torch.equal(a, c)


def test_exact_split_batch_and_graph():
    g = scene.make_gaussians(150_000, 3, seed=43)
    views = scene.make_batched_views(8, seed=7, radius=(3.0, 6.0),
                                     resolutions=((320, 240), (640, 480), (272, 400), (800, 720)))
    gt = F.gaussians_to_torch(g, DEV)
    vf = ["none", ("rings", 0.15, 0.4), None, "none", ("rings", 0.3, 0.6), None, "none", None]
    st = [F.settings_from_view(v, K=8, active_sh_bases=16) for v in views]
    r = F.Renderer(DEV)
    exact = [x.clone() for x in r.render(*gt, st, view_foveation=vf)]
    r.set_blend_split(0.1, 0, exact=True)
    split = [x.clone() for x in r.render(*gt, st, view_foveation=vf)]
    assert r.blend_split_stats()["split_tiles"] > 0
    graph = r.capture(*gt, st, view_foveation=vf, capacity_headroom=2.0)
    replay = graph.launch(sync=True)
    for a, b, c in zip(exact, split, replay):
        assert torch.equal(a, b) and torch.equal(a, c)
    graph.close()
    r.close()
