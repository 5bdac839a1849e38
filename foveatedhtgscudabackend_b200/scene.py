"""Seeded synthetic scenes, cameras and tile masks for the foveated HTGS renderer.

The reference renderer receives Gaussians that are already *activated* (linear scales,
post-sigmoid opacities, rotations used as (w, x, y, z) without renormalisation,
`rasterization/include/utils/kernel_utils.cuh:76-137`) and camera/mask tensors that an
external framework precomputes (`torch_bindings/rasterization.py:22-43`).  This module builds
all of them from a seed, with the distributions of the benchmark configurations:

* means ~ N(0,1)^3, rescaled so that max |coordinate| = 2 (a 4-unit box);
* scales = exp(N(-4.5, 0.5)), quaternions = normalised N(0,1)^4, opacity = sigmoid(N(0,1.5));
* SH DC ~ N(0, 0.3), higher bands ~ N(0, 0.05) (`sh_rest` is [N, S, 3], S = 0/3/8/15);
* pinhole camera, vertical field of view 60 degrees, at (0,0,-6) looking at the origin,
  near 0.2 / far 100; stereo eyes offset by +-IPD/2 along the camera's x axis;
* visibility bitmask over the 16x16 "large" tile grid, its summed-area table
  ((gx+1)*(gy+1) entries, leading zero row/column, read at `kernel_utils.cuh:184-198`) and
  the 49x49 fovea summed-area table that counts the three extra sub-tiles of every tile of
  the 48x48 window whose centre lies inside the 24-tile fovea circle
  (`kernel_utils.cuh:61-73,168-210`).

Everything here is NumPy on the host; the torch conversion lives in `settings_to_torch`.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TILE_LARGE = 16
TILE_SMALL = 8
FOVEATION_RADIUS_TILES = 24  # (375 + 15) // 16, rasterization/include/config.h:30-31
FOVEA_TABLE_SIDE = 2 * FOVEATION_RADIUS_TILES + 1  # 49

SH_BASES_FOR_DEGREE = {0: 1, 1: 4, 2: 9, 3: 16}


@dataclass
class Gaussians:
    positions: np.ndarray  # [N,3] f32
    scales: np.ndarray  # [N,3] f32 (activated)
    rotations: np.ndarray  # [N,4] f32 (w,x,y,z), unit
    opacities: np.ndarray  # [N,1] f32 (activated)
    sh_0: np.ndarray  # [N,1,3] f32
    sh_rest: np.ndarray  # [N,S,3] f32

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])

    @property
    def sh_degree(self) -> int:
        s = self.sh_rest.shape[1] + 1
        return {1: 0, 4: 1, 9: 2, 16: 3}[s]


@dataclass
class View:
    """One camera with everything the reference's RasterizerSettings carries."""

    width: int
    height: int
    focal_x: float
    focal_y: float
    center_x: float
    center_y: float
    near_plane: float
    far_plane: float
    M: np.ndarray  # [3,4] world -> view
    VPM: np.ndarray  # [4,4] world -> screen (homogeneous)
    VPR_inv: np.ndarray  # [4,4] screen -> world direction
    cam_position: np.ndarray  # [3]
    gaze_position: np.ndarray  # [2] pixels
    visibility_mask: np.ndarray  # uint32 words
    visibility_mask_area_table: np.ndarray  # uint32 [(gy+1)*(gx+1)]
    fovea_mask_area_table: np.ndarray  # uint32 [49*49]
    extra: dict = field(default_factory=dict)

    @property
    def grid_large(self) -> tuple[int, int]:
        return (-(-self.width // TILE_LARGE), -(-self.height // TILE_LARGE))


def make_gaussians(n: int, sh_degree: int = 3, seed: int = 0) -> Gaussians:
    """Synthetic Gaussians with the benchmark distributions (activated parameters)."""
    rng = np.random.default_rng(seed)
    pos = rng.standard_normal((n, 3))
    if n > 0:
        pos = pos / max(np.abs(pos).max(), 1e-12) * 2.0
    log_scales = rng.normal(-4.5, 0.5, size=(n, 3))
    q = rng.standard_normal((n, 4))
    q /= np.maximum(np.linalg.norm(q, axis=1, keepdims=True), 1e-12)
    opac = 1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.5, size=(n, 1))))
    dc = rng.normal(0.0, 0.3, size=(n, 1, 3))
    n_rest = SH_BASES_FOR_DEGREE[sh_degree] - 1
    rest = rng.normal(0.0, 0.05, size=(n, n_rest, 3))
    f32 = np.float32
    return Gaussians(
        positions=np.ascontiguousarray(pos, f32),
        scales=np.ascontiguousarray(np.exp(log_scales), f32),
        rotations=np.ascontiguousarray(q, f32),
        opacities=np.ascontiguousarray(opac, f32),
        sh_0=np.ascontiguousarray(dc, f32),
        sh_rest=np.ascontiguousarray(rest, f32),
    )


def look_at(position, target, up=(0.0, -1.0, 0.0)) -> np.ndarray:
    """World->view rotation rows (right, down, forward); image y grows downwards."""
    p = np.asarray(position, np.float64)
    fw = np.asarray(target, np.float64) - p
    fw /= np.linalg.norm(fw)
    r = np.cross(fw, np.asarray(up, np.float64))
    if np.linalg.norm(r) < 1e-9:
        r = np.cross(fw, np.array([1.0, 0.0, 0.0]))
    r /= np.linalg.norm(r)
    dn = np.cross(fw, r)
    return np.stack([r, dn, fw])


def visibility_tables(grid_w: int, grid_h: int, visible: np.ndarray | None = None):
    """Bitmask words + summed-area table for a [grid_h, grid_w] boolean visibility map."""
    if visible is None:
        visible = np.ones((grid_h, grid_w), bool)
    visible = np.asarray(visible, bool)
    assert visible.shape == (grid_h, grid_w)
    flat = visible.reshape(-1)
    n_words = (flat.size + 31) // 32
    words = np.zeros(n_words, np.uint64)
    idx = np.nonzero(flat)[0]
    np.add.at(words, idx // 32, (np.uint64(1) << (idx % 32).astype(np.uint64)))
    words = words.astype(np.uint32)
    sat = np.zeros((grid_h + 1, grid_w + 1), np.uint32)
    sat[1:, 1:] = np.cumsum(np.cumsum(visible.astype(np.uint32), 0), 1)
    return words, sat.reshape(-1)


def fovea_table() -> np.ndarray:
    """49x49 SAT counting 3 extra sub-tiles for window tiles inside the fovea circle.

    Window tile (i, j) is tile (gaze_x - 24 + i, gaze_y - 24 + j); its centre is inside the
    fovea when (i - 24 + 0.5)^2 + (j - 24 + 0.5)^2 < 24^2, evaluated in float32 exactly as
    `is_in_fovea` does (`kernel_utils.cuh:61-73`).
    """
    r = FOVEATION_RADIUS_TILES
    i = np.arange(2 * r, dtype=np.float32)
    d = (i - np.float32(r) + np.float32(0.5)).astype(np.float32)
    inside = (d[None, :] * d[None, :] + d[:, None] * d[:, None]).astype(np.float32) < np.float32(r * r)
    cnt = inside.astype(np.uint32) * 3
    sat = np.zeros((2 * r + 1, 2 * r + 1), np.uint32)
    sat[1:, 1:] = np.cumsum(np.cumsum(cnt, 0), 1)
    return sat.reshape(-1)


def make_view(
    width: int,
    height: int,
    position=(0.0, 0.0, -6.0),
    target=(0.0, 0.0, 0.0),
    fov_y_deg: float = 60.0,
    near: float = 0.2,
    far: float = 100.0,
    eye_offset: float = 0.0,
    gaze_ndc=(0.0, 0.0),
    visible: np.ndarray | None = None,
    up=(0.0, -1.0, 0.0),
) -> View:
    """Pinhole view; `eye_offset` shifts the eye along the camera's x axis (stereo)."""
    R = look_at(position, target, up)
    pos = np.asarray(position, np.float64) + eye_offset * R[0]
    t = -R @ pos
    fy = (height / 2.0) / math.tan(math.radians(fov_y_deg) / 2.0)
    fx = fy
    cx, cy = width / 2.0, height / 2.0
    M = np.concatenate([R, t[:, None]], 1)
    a = (far + near) / (far - near)
    b = -2.0 * far * near / (far - near)
    P = np.array([[fx, 0, cx, 0], [0, fy, cy, 0], [0, 0, a, b], [0, 0, 1, 0]], np.float64)
    M4 = np.concatenate([M, [[0, 0, 0, 1]]], 0)
    VPM = P @ M4
    Kinv = np.array([[1 / fx, 0, -cx / fx], [0, 1 / fy, -cy / fy], [0, 0, 1]], np.float64)
    VPR_inv = np.zeros((4, 4))
    VPR_inv[:3, :3] = R.T @ Kinv
    VPR_inv[3, 3] = 1.0
    gx, gy = -(-width // TILE_LARGE), -(-height // TILE_LARGE)
    words, sat = visibility_tables(gx, gy, visible)
    gaze = np.array([(0.5 + 0.5 * gaze_ndc[0]) * width, (0.5 + 0.5 * gaze_ndc[1]) * height], np.float32)
    f32 = np.float32
    return View(
        width=int(width), height=int(height),
        focal_x=float(fx), focal_y=float(fy), center_x=float(cx), center_y=float(cy),
        near_plane=float(near), far_plane=float(far),
        M=M.astype(f32), VPM=VPM.astype(f32), VPR_inv=VPR_inv.astype(f32),
        cam_position=pos.astype(f32), gaze_position=gaze,
        visibility_mask=words, visibility_mask_area_table=sat,
        fovea_mask_area_table=fovea_table(),
    )


def make_stereo_views(width: int, height: int, ipd: float = 0.063, gaze_sigma: float = 0.05,
                      seed: int = 0, **kw) -> tuple[View, View]:
    """Left/right eyes at -/+ ipd/2 along camera x; gaze = centre + N(0, sigma) in NDC."""
    rng = np.random.default_rng(seed + 7919)
    g = rng.normal(0.0, gaze_sigma, size=2)
    left = make_view(width, height, eye_offset=-ipd / 2, gaze_ndc=g, **kw)
    right = make_view(width, height, eye_offset=+ipd / 2, gaze_ndc=g, **kw)
    return left, right


BATCH_RESOLUTIONS = ((640, 480), (1280, 720), (1920, 1080), (2064, 2208))


def make_batched_views(n_views: int = 64, seed: int = 0, radius=(4.0, 8.0), resolutions=BATCH_RESOLUTIONS,
                       gaze_range: float = 0.8) -> list[View]:
    """Cameras on a sphere around the origin looking at it, for batched rendering.

    Directions uniform on the sphere (away from the poles, where the fixed up vector
    degenerates), distance uniform in `radius`, resolution drawn uniformly from `resolutions`,
    gaze uniform in [-gaze_range, gaze_range]^2 NDC per view.
    """
    rng = np.random.default_rng(seed + 104729)
    views = []
    for _ in range(n_views):
        while True:
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            if abs(d[1]) < 0.95:
                break
        r = rng.uniform(*radius)
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        g = rng.uniform(-gaze_range, gaze_range, size=2)
        views.append(make_view(w, h, position=tuple(r * d), gaze_ndc=tuple(g)))
    return views


SERVED_RESOLUTIONS = ((1440, 1584), (2064, 2208))


def make_served_requests(duration_s: float, rate_hz: float, n_scenes: int, seed: int = 0,
                         resolutions=SERVED_RESOLUTIONS, radius=(4.0, 8.0), ipd: float = 0.063,
                         gaze_sigma: float = 0.1) -> list[tuple[float, int, View, View]]:
    """A request stream: (arrival s, scene index, left eye, right eye) sorted by arrival.

    Arrivals are Poisson at `rate_hz` over `duration_s`; each request draws its scene uniformly,
    one resolution (both eyes) uniformly from `resolutions`, a head position uniform on the
    sphere (away from the poles) at a distance uniform in `radius` looking at the origin, and a
    gaze of N(0, gaze_sigma) NDC shared by both eyes (eyes at -/+ ipd/2 along the head's x).
    """
    rng = np.random.default_rng(seed + 7727)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            return out
        si = int(rng.integers(n_scenes))
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        while True:
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            if abs(d[1]) < 0.95:
                break
        pos = tuple(rng.uniform(*radius) * d)
        g = tuple(np.clip(rng.normal(0.0, gaze_sigma, size=2), -0.95, 0.95))
        left = make_view(w, h, position=pos, eye_offset=-ipd / 2, gaze_ndc=g)
        right = make_view(w, h, position=pos, eye_offset=+ipd / 2, gaze_ndc=g)
        out.append((t, si, left, right))


def random_visibility(grid_w: int, grid_h: int, p_visible: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.random((grid_h, grid_w)) < p_visible


def lens_visibility(grid_w: int, grid_h: int) -> np.ndarray:
    """Elliptical lens mask: tiles whose centre lies in the inscribed ellipse are visible."""
    y, x = np.mgrid[0:grid_h, 0:grid_w]
    u = (x + 0.5) / grid_w * 2 - 1
    v = (y + 0.5) / grid_h * 2 - 1
    return (u * u + v * v) <= 1.0


def sh_background(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed + 31)
    return rng.normal(0.0, 0.5, size=(16, 3)).astype(np.float32)


def texture_background(w: int = 64, h: int = 32, seed: int = 0, raw: bool = False) -> np.ndarray:
    rng = np.random.default_rng(seed + 57)
    t = rng.random((3, h, w)).astype(np.float32)
    if raw:
        t = (t * 6.0 - 3.0).astype(np.float32)
    return t
