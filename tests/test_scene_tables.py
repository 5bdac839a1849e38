"""Host logic: synthetic inputs, area tables and tile geometry (no GPU)."""
import numpy as np
import pytest

from foveatedhtgscudabackend_b200 import scene
import oracle as O


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_visibility_sat_matches_brute_force(seed):
    gw, gh = 23, 17
    vis = scene.random_visibility(gw, gh, 0.7, seed)
    words, sat = scene.visibility_tables(gw, gh, vis)
    sat = sat.reshape(gh + 1, gw + 1)
    for _ in range(200):
        rng = np.random.default_rng(seed)
        x0, x1 = sorted(rng.integers(0, gw + 1, 2))
        y0, y1 = sorted(rng.integers(0, gh + 1, 2))
        n = int(sat[y1, x1]) + int(sat[y0, x0]) - int(sat[y0, x1]) - int(sat[y1, x0])
        assert n == int(vis[y0:y1, x0:x1].sum())
    flat = vis.reshape(-1)
    for t in range(flat.size):
        assert bool(words[t // 32] >> (t % 32) & 1) == bool(flat[t])


def test_fovea_table_counts_three_per_inside_tile():
    sat = scene.fovea_table().reshape(49, 49)
    r = 24
    inside = 0
    for j in range(48):
        for i in range(48):
            dx = np.float32(i - r) + np.float32(0.5)
            dy = np.float32(j - r) + np.float32(0.5)
            inside += bool(np.float32(dx * dx + dy * dy) < np.float32(r * r))
    assert int(sat[48, 48]) == 3 * inside
    assert np.array_equal(sat, sat.T)


# Key widths at the benchmark resolutions (tile-only keys, end_bit = bit_width(T + 1)).
@pytest.mark.parametrize("w,h,T_L,end_bit", [(640, 480, 1200, 13), (1280, 720, 3600, 14), (1920, 1080, 8160, 15),
                                             (1440, 1584, 8910, 16), (2064, 2208, 17802, 17)])
def test_grid_geometry(w, h, T_L, end_bit):
    v = scene.make_view(w, h)
    geo = O.geometry(v)
    assert geo["grid_large_w"] * geo["grid_large_h"] == T_L
    assert geo["n_tiles"] == 4 * T_L
    assert geo["end_bit"] == end_bit


@pytest.mark.parametrize("gaze,expect", [((0.0, 0.0), (0, 0)), ((7.9, 8.0), (0, 1)), ((-50, 1e6), (0, 30)),
                                         ((639.0, 479.0), (40, 30))])
def test_gaze_tile_rounding_and_clamp(gaze, expect):
    v = scene.make_view(640, 480)
    v.gaze_position = np.asarray(gaze, np.float32)
    geo = O.geometry(v)
    assert (geo["gaze_tile_x"], geo["gaze_tile_y"]) == expect


def test_generator_distributions_and_determinism():
    a = scene.make_gaussians(5000, 3, seed=3)
    b = scene.make_gaussians(5000, 3, seed=3)
    assert all(np.array_equal(getattr(a, k), getattr(b, k)) for k in ("positions", "scales", "rotations", "sh_rest"))
    assert np.abs(a.positions).max() == pytest.approx(2.0)
    assert np.allclose(np.linalg.norm(a.rotations, axis=1), 1.0, atol=1e-6)
    assert 0.0 < a.opacities.min() and a.opacities.max() < 1.0
    assert a.sh_rest.shape == (5000, 15, 3)
    assert abs(np.log(a.scales).mean() + 4.5) < 0.05
    assert scene.make_gaussians(10, 0).sh_rest.shape == (10, 0, 3)


def test_stereo_views_offset_along_camera_x():
    L, R = scene.make_stereo_views(2064, 2208, ipd=0.063, seed=0)
    d = R.cam_position - L.cam_position
    assert np.allclose(d, [0.063, 0.0, 0.0], atol=1e-6)
    assert np.allclose(L.gaze_position, R.gaze_position)
