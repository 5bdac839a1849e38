"""Known-answer and property tests of the CPU oracle (no GPU)."""
import numpy as np
import pytest

from foveatedhtgscudabackend_b200 import scene
import oracle as O


def one_gaussian(pos=(0.0, 0.0, 0.0), scale=0.05, opacity=0.9, dc=(0.5, -0.2, 0.1)):
    C0 = 0.28209479177387814
    g = scene.make_gaussians(1, 0, seed=0)
    g.positions[:] = np.asarray(pos, np.float32)
    g.scales[:] = np.float32(scale)
    g.rotations[:] = np.asarray([1, 0, 0, 0], np.float32)
    g.opacities[:] = np.float32(opacity)
    g.sh_0[:] = np.asarray(dc, np.float32)
    rgb = 0.5 + C0 * np.asarray(dc, np.float64)
    return g, rgb


def test_empty_scene_is_background():
    g = scene.make_gaussians(0, 3)
    v = scene.make_view(320, 240)
    img = O.render(g, v, K=8, precision=64)
    assert not img.any()
    bg = scene.sh_background(0)
    img = O.render(g, v, K=8, precision=64, background=bg, background_type=1)
    assert img.max() > 0.0


@pytest.mark.parametrize("precision", [32, 64])
def test_single_gaussian_centre_pixel_known_answer(precision):
    # A Gaussian whose mean projects exactly onto pixel (160, 120): alpha = opacity there, the
    # fragment is the only core entry, colour = RGBA8-quantised premultiplied colour.
    g, rgb = one_gaussian()
    v = scene.make_view(320, 240, gaze_ndc=(0.0, 0.0))
    img = O.render(g, v, K=4, precision=precision, active_sh_bases=1)
    px = img[:, 120, 160].astype(np.float64)
    q = np.floor(np.clip(rgb * 0.9, 0, 1) * 255.0 + 0.5) / 255.0
    assert np.allclose(px, q, atol=1e-6)
    assert img[:, 0, 0].max() == 0.0 and img[:, 239, 319].max() == 0.0


def test_sub_threshold_opacity_contributes_nothing_but_creates_instances():
    g, _ = one_gaussian(opacity=0.003)
    v = scene.make_view(320, 240)
    img, inter = O.render(g, v, K=4, precision=64, active_sh_bases=1, intermediates=True)
    assert not img.any()
    assert inter["n_instances"] >= 0


def test_near_plane_culls_gaussian_behind_camera():
    g, _ = one_gaussian(pos=(0.0, 0.0, -7.0))
    v = scene.make_view(320, 240)
    pr = O.preprocess(g, v, K=4, precision=32, active_sh_bases=1)
    assert pr["n_touched"][0] == 0


def test_instances_sorted_stable_and_ranges_consistent():
    g = scene.make_gaussians(3000, 1, seed=4)
    v = scene.make_view(480, 400, gaze_ndc=(0.4, 0.3), visible=scene.random_visibility(30, 25, 0.8, 1))
    _, inter = O.render(g, v, K=8, precision=32, active_sh_bases=4, intermediates=True)
    keys, vals = inter["keys"], inter["values"]
    sent = 0xFFFF
    valid = keys != sent
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    # stable: within a key, primitive indices ascend
    same = (keys[1:] == keys[:-1]) & valid[1:]
    assert np.all(vals[1:][same] > vals[:-1][same])
    r = inter["instance_ranges"]
    for t in np.unique(keys[valid]):
        idx = np.flatnonzero(keys == t)
        assert (r[t, 0], r[t, 1]) == (idx[0], idx[-1] + 1)
    # fovea large tiles carry 4 identical sub-tile lists
    tm = inter["tile_index_map_partitioned"]
    ty = inter["tile_type_partitioned"]
    for e in tm[ty == 0][::4][:20]:
        base = (e // 4) * 4
        lists = [vals[r[base + i, 0]:r[base + i, 1]] for i in range(4)]
        assert all(np.array_equal(lists[0], l) for l in lists[1:])


def test_partition_ranges_single_active_tile_quirk():
    # exactly one visible periphery tile: the reference's range kernel starts at index 1, so
    # all partition ranges stay zero and nothing is blended.
    vis = np.zeros((30, 40), bool)
    vis[29, 39] = True
    v = scene.make_view(640, 480, gaze_ndc=(-1.0, -1.0), visible=vis)
    t = O.classify(v)
    assert t["n_active_tiles"] == 1
    assert not t["partition_ranges"].any()


@pytest.mark.parametrize("K", [1, 2, 4, 8, 16, 32])
def test_k_variants_images_valid(K):
    g = scene.make_gaussians(2000, 2, seed=K)
    v = scene.make_view(256, 192, gaze_ndc=(0.2, -0.1))
    img = O.render(g, v, K=K, precision=32, active_sh_bases=9)
    assert np.isfinite(img).all() and img.min() >= 0.0 and img.max() <= 1.0 and img.max() > 0.0


def test_fp32_restatement_close_to_fp64():
    g = scene.make_gaussians(6000, 3, seed=9)
    v = scene.make_view(640, 480, gaze_ndc=(0.3, -0.2))
    a = O.render(g, v, K=8, precision=32)
    b = O.render(g, v, K=8, precision=64)
    mse = float(np.mean((a.astype(np.float64) - b) ** 2))
    assert 10 * np.log10(1.0 / max(mse, 1e-30)) > 45.0


@pytest.mark.parametrize("blur", [False, True])
@pytest.mark.parametrize("chw", [False, True])
def test_layouts_and_blur_consistent(blur, chw):
    g = scene.make_gaussians(3000, 3, seed=1)
    v = scene.make_view(400, 320, gaze_ndc=(-0.6, -0.6))
    img = O.render(g, v, K=8, precision=32, to_chw=chw, blur=blur)
    ref = O.render(g, v, K=8, precision=32, to_chw=True, blur=blur)
    if not chw:
        img = np.transpose(img, (2, 0, 1))
    assert np.array_equal(img, ref)
