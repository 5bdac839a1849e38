"""NumPy restatement of the overlays, tile masks and display packing — TEST INFRASTRUCTURE ONLY.

Only the test-suite and the golden-fixture script use this module, as the checker of the
device kernels in libfhtgs.so (csrc/fhtgs_extras.cu).  Parity of the two overlays is pinned by
tests/golden/visualization_reference.npz, written by the reference's own `_C_visualization`
module (tests/golden/make_golden_visualization.py).

* `visualize_gaze`            — visualization/include/kernels/visualization.cuh:11-50 and
                                visualization/src/visualization.cu:27-57
* `visualize_tile_boundaries` — visualization.cuh:52-111, visualization.cu:60-236, with the tile
                                classes of rasterization/include/kernels/shared_kernels.cuh:155-237
                                and rasterization/include/utils/kernel_utils.cuh:43-58
* `tile_masks`                — the mask layout read at kernel_utils.cuh:168-210 (no reference
                                builder: the reference takes the masks precomputed)
* `pack_display`              — no reference counterpart; the packing rule of include/fhtgs.h
"""
from __future__ import annotations

import numpy as np

TILE_SMALL = 8
TILE_LARGE = 16
FOVEATION_RADIUS_TILES = 24
BLEND_RADIUS_TILES = 15

ORANGE = np.array([0.902, 0.624, 0.0], np.float32)  # fovea sub-tiles (visualization.cu:190)
LIGHT_BLUE = np.array([0.337, 0.706, 0.914], np.float32)  # blended sub-tiles (visualization.cu:205)
GREEN = np.array([0.0, 0.620, 0.451], np.float32)  # periphery tiles (visualization.cu:220)


def _image_wh(image: np.ndarray, to_chw: bool) -> tuple[int, int]:
    return (image.shape[2], image.shape[1]) if to_chw else (image.shape[1], image.shape[0])


def _put(image: np.ndarray, xs: np.ndarray, ys: np.ndarray, color, to_chw: bool) -> None:
    c = np.asarray(color, np.float32)
    if to_chw:
        for k in range(3):
            image[k, ys, xs] = c[k]
    else:
        image[ys, xs, :] = c


def _clamp_gaze(gaze, w: int, h: int) -> tuple[np.float32, np.float32]:
    g = np.asarray(gaze, np.float32).reshape(-1)
    return (np.float32(min(max(g[0], np.float32(0)), np.float32(w - 1))),
            np.float32(min(max(g[1], np.float32(0)), np.float32(h - 1))))


def visualize_gaze(image: np.ndarray, gaze, color, size: int, vtype: int, to_chw: bool) -> np.ndarray:
    """Marker of `size` px at the clamped gaze: 0 circle, 2 cross, other types a square.

    Thread (X, Y) of the (ceil(size/8)*8)^2 launch takes offset trunc(float(X) - size/2) (float
    arithmetic, truncation toward zero) and skips when the offset exceeds size/2 in float, when
    off the circle (x^2 + y^2 > (size/2)^2, int sum compared in float) or off the cross
    (|x| > 1 and |y| > 1); the pixel is int(gaze) + offset, inside the image.
    """
    w, h = _image_wh(image, to_chw)
    if size <= 0:
        return image
    gx, gy = _clamp_gaze(gaze, w, h)
    half = np.float32(np.float32(size) / np.float32(2))
    n = -(-size // TILE_SMALL) * TILE_SMALL
    idx = np.arange(n, dtype=np.float32)
    off = np.trunc((idx - half).astype(np.float32)).astype(np.int64)
    xo, yo = np.meshgrid(off, off, indexing="xy")
    keep = (xo.astype(np.float32) <= half) & (yo.astype(np.float32) <= half)
    if vtype == 0:
        keep &= (xo * xo + yo * yo).astype(np.float32) <= np.float32(half * half)
    elif vtype == 2:
        keep &= ~((np.abs(xo) > 1) & (np.abs(yo) > 1))
    x = int(gx) + xo
    y = int(gy) + yo
    keep &= (x >= 0) & (x < w) & (y >= 0) & (y < h)
    _put(image, x[keep], y[keep], color, to_chw)
    return image


def _in_circle(tx, ty, g, radius: int):
    dx = (np.asarray(tx, np.float32) + np.float32(0.5)) - g[0]
    dy = (np.asarray(ty, np.float32) + np.float32(0.5)) - g[1]
    return (dx * dx + dy * dy).astype(np.float32) < np.float32(radius * radius)


def _border(tw: int, th: int) -> tuple[np.ndarray, np.ndarray]:
    """Border pixels of a tw x th rectangle in the reference's thread order (visualization.cuh:73-91)."""
    xs, ys = [], []
    for k in range(2 * tw + 2 * th - 4):
        if k < tw:
            x, y = k, 0
        elif k < 2 * tw:
            x, y = k - tw, th - 1
        elif k < 2 * tw + th - 2:
            x, y = 0, k - 2 * tw + 1
        else:
            x, y = tw - 1, k - (2 * tw + th - 2) + 1
        xs.append(x)
        ys.append(y)
    return np.asarray(xs), np.asarray(ys)


def visualize_tile_boundaries(image: np.ndarray, visibility_mask: np.ndarray, gaze, to_chw: bool) -> np.ndarray:
    """Outlines each visible large tile by its class for the gaze.

    The gaze is rounded to the nearest large-tile corner, (int(g) + 8) // 16, and clamped to the
    SMALL-tile grid width/height minus one (visualization.cu:84-92, as the reference does).
    A visible tile whose centre lies inside the 24-tile circle is split into four 8x8 sub-tiles,
    orange inside the 15-tile circle and light blue outside it; other visible tiles get a green
    16x16 border.  When at most one sub-tile entry is active in total the reference's partition
    ranges stay zero and nothing is drawn (shared_kernels.cuh:222-236).
    """
    w, h = _image_wh(image, to_chw)
    gx, gy = _clamp_gaze(gaze, w, h)
    glw, glh = -(-w // TILE_LARGE), -(-h // TILE_LARGE)
    gsw, gsh = 2 * glw, 2 * glh
    g = (np.float32(max(0, min(gsw - 1, (int(gx) + TILE_LARGE // 2) // TILE_LARGE))),
         np.float32(max(0, min(gsh - 1, (int(gy) + TILE_LARGE // 2) // TILE_LARGE))))
    n = glw * glh
    words = np.asarray(visibility_mask, np.uint32).reshape(-1)
    t = np.arange(n)
    vis = ((words[t // 32] >> (t % 32).astype(np.uint32)) & 1).astype(bool)
    tx, ty = t % glw, t // glw
    fovea = _in_circle(tx, ty, g, FOVEATION_RADIUS_TILES)
    inner = _in_circle(tx, ty, g, BLEND_RADIUS_TILES)
    n_active = int(np.sum(np.where(vis, np.where(fovea, 4, 1), 0)))
    if n_active <= 1:
        return image
    bs_x, bs_y = _border(TILE_SMALL, TILE_SMALL)
    bl_x, bl_y = _border(TILE_LARGE, TILE_LARGE)
    for tile in t[vis]:
        ox, oy = int(tx[tile]) * TILE_LARGE, int(ty[tile]) * TILE_LARGE
        if fovea[tile]:
            color = ORANGE if inner[tile] else LIGHT_BLUE
            for sub in range(4):
                xs = ox + (sub % 2) * TILE_SMALL + bs_x
                ys = oy + (sub // 2) * TILE_SMALL + bs_y
                m = (xs < w) & (ys < h)
                _put(image, xs[m], ys[m], color, to_chw)
        else:
            xs, ys = ox + bl_x, oy + bl_y
            m = (xs < w) & (ys < h)
            _put(image, xs[m], ys[m], GREEN, to_chw)
    return image


def tile_masks(width: int, height: int, visible: np.ndarray | None = None):
    """(bit words, (gw+1)x(gh+1) summed-area table, 49x49 fovea table), by plain loops."""
    gw, gh = -(-width // TILE_LARGE), -(-height // TILE_LARGE)
    vis = np.ones((gh, gw), bool) if visible is None else (np.asarray(visible).reshape(gh, gw) != 0)
    words = [0] * (-(-(gw * gh) // 32))
    for t in range(gw * gh):
        if vis[t // gw, t % gw]:
            words[t // 32] |= 1 << (t % 32)
    sat = np.zeros((gh + 1, gw + 1), np.uint64)
    for y in range(gh):
        row = 0
        for x in range(gw):
            row += int(vis[y, x])
            sat[y + 1, x + 1] = sat[y, x + 1] + row
    r = FOVEATION_RADIUS_TILES
    fov = np.zeros((2 * r + 1, 2 * r + 1), np.uint64)
    for j in range(2 * r):
        row = 0
        for i in range(2 * r):
            d = (np.float32(i - r) + np.float32(0.5), np.float32(j - r) + np.float32(0.5))
            row += 3 if np.float32(d[0] * d[0] + d[1] * d[1]) < np.float32(r * r) else 0
            fov[j + 1, i + 1] = fov[j, i + 1] + row
    return (np.asarray(words, np.uint64).astype(np.uint32), sat.reshape(-1).astype(np.uint32),
            fov.reshape(-1).astype(np.uint32))


def pack_display(images, to_chw: bool = True, bgra: bool = False) -> np.ndarray:
    """[H, n*W, 4] uint8: clamp to [0,1] (NaN -> 0), trunc(fma(c, 255, 0.5)) per channel, alpha 255."""
    planes = []
    for im in images:
        im = np.asarray(im, np.float32)
        hwc = np.transpose(im, (1, 2, 0)) if to_chw else im
        c = np.fmin(np.fmax(hwc, np.float32(0)), np.float32(1))
        # exact c*255 + 0.5 in float64, one rounding to float32 (the fused multiply-add), truncate
        q = np.trunc((c.astype(np.float64) * 255.0 + 0.5).astype(np.float32)).astype(np.uint8)
        if bgra:
            q = q[..., ::-1]
        planes.append(np.concatenate([q, np.full(q.shape[:2] + (1,), 255, np.uint8)], axis=2))
    return np.concatenate(planes, axis=1)
