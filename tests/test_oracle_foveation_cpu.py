"""CPU tests of the oracle's ring and no-foveation modes (restatements of the product's
FHTGS_FOVEATION_RINGS / _NONE; the reference has neither, so these pin the oracle by
properties: limits of the ring radii, agreement with the reference mode where both render the
same tiles at full resolution, and exact reproduction of linear colour ramps by the strided
bilinear fill)."""
import numpy as np
import pytest

from foveatedhtgscudabackend_b200 import scene
import oracle as O

W, H = 200, 136  # ragged: 13 x 9 large tiles, the last column/row partial


@pytest.fixture(scope="module")
def g():
    return scene.make_gaussians(6000, 1, seed=5)


def tile_types(v):
    """Reference-mode classes of the large tiles: 0 fovea, 2 blended, 1 periphery."""
    geo = O.geometry(v)
    gw, gh = geo["grid_large_w"], geo["grid_large_h"]
    gx, gy = geo["gaze_tile_x"], geo["gaze_tile_y"]
    out = np.ones((gh, gw), np.int8)
    for ty in range(gh):
        for tx in range(gw):
            d2 = (np.float32(tx) + np.float32(0.5) - np.float32(gx)) ** 2 + (np.float32(ty) + np.float32(0.5) - np.float32(gy)) ** 2
            out[ty, tx] = 0 if d2 < 15 * 15 else 2 if d2 < 24 * 24 else 1
    return out


@pytest.mark.parametrize("precision", [32, 64])
def test_rings_with_large_radii_equal_no_foveation(g, precision):
    v = scene.make_view(W, H, gaze_ndc=(0.3, -0.2))
    none = O.render(g, v, K=8, active_sh_bases=4, precision=precision, foveation="none")
    full = O.render(g, v, K=8, active_sh_bases=4, precision=precision, foveation="rings", rings=(3.0, 3.0))
    assert np.array_equal(none, full)
    assert none.max() > 0.0


def test_no_foveation_matches_reference_on_its_fovea_tiles(g):
    v = scene.make_view(W, H, gaze_ndc=(-0.1, 0.2))
    ref = O.render(g, v, K=8, active_sh_bases=4, precision=64)
    none = O.render(g, v, K=8, active_sh_bases=4, precision=64, foveation="none")
    types = tile_types(v)
    px_types = np.repeat(np.repeat(types, 16, 0), 16, 1)[:H, :W]
    fov = px_types == 0
    assert fov.any()
    assert np.array_equal(ref[:, fov], none[:, fov])


def test_strided_samples_equal_the_full_resolution_pixels(g):
    """Every ring renders its sample positions with the per-pixel arithmetic of a full tile."""
    v = scene.make_view(W, H, gaze_ndc=(0.0, 0.0))
    none = O.render(g, v, K=8, active_sh_bases=4, precision=64, foveation="none")
    quarter = O.render(g, v, K=8, active_sh_bases=4, precision=64, foveation="rings", rings=(0.0, 0.0))
    half = O.render(g, v, K=8, active_sh_bases=4, precision=64, foveation="rings", rings=(0.0, 3.0))
    assert np.array_equal(quarter[:, ::4, ::4], none[:, ::4, ::4])
    assert np.array_equal(half[:, ::2, ::2], none[:, ::2, ::2])
    assert not np.array_equal(quarter, none)


def test_ring_levels_follow_the_ndc_radii(g):
    """With only the inner disc at full resolution, pixels there equal the unfoveated image and
    the 2x/4x rings differ from it (they are interpolated)."""
    v = scene.make_view(W, H, gaze_ndc=(0.0, 0.0))
    none = O.render(g, v, K=8, active_sh_bases=4, precision=64, foveation="none")
    rings = O.render(g, v, K=8, active_sh_bases=4, precision=64, foveation="rings", rings=(0.25, 0.6))
    gx, gy = v.gaze_position
    for ty in range(-(-H // 16)):
        for tx in range(-(-W // 16)):
            cx, cy = np.float32(tx * 16 + 8), np.float32(ty * 16 + 8)
            dx = (cx - np.float32(min(max(gx, 0), W - 1))) / np.float32(0.5 * W)
            dy = (cy - np.float32(min(max(gy, 0), H - 1))) / np.float32(0.5 * H)
            r2 = np.float32(dx * dx) + np.float32(dy * dy)
            sl = (slice(None), slice(ty * 16, min(H, ty * 16 + 16)), slice(tx * 16, min(W, tx * 16 + 16)))
            if r2 < np.float32(0.25) * np.float32(0.25):
                assert np.array_equal(rings[sl], none[sl]), (tx, ty)


def test_quarter_fill_is_bilinear_between_the_samples(g):
    """All tiles at 4x: every pixel between samples is the bilinear mix of the four samples
    around it (interior tiles, all tiles visible), clamped to [0, 1]."""
    v = scene.make_view(W, H, gaze_ndc=(0.0, 0.0))
    q = O.render(g, v, K=8, active_sh_bases=4, precision=64, foveation="rings", rings=(0.0, 0.0))
    s = q[:, ::4, ::4].astype(np.float64)
    f = (np.arange(4) / 4.0)
    for y in range(0, (H // 16 - 1) * 16):
        for x in range(0, (W // 16 - 1) * 16):
            if x % 4 == 0 and y % 4 == 0:
                continue
            bx, by, xf, yf = x // 4, y // 4, f[x % 4], f[y % 4]
            e = (s[:, by, bx] * (1 - xf) * (1 - yf) + s[:, by, bx + 1] * xf * (1 - yf)
                 + s[:, by + 1, bx] * (1 - xf) * yf + s[:, by + 1, bx + 1] * xf * yf)
            assert np.allclose(q[:, y, x], np.clip(e, 0, 1), atol=2e-6), (x, y)
