"""ctypes front end of the CPU oracle (oracle/fhtgs_oracle.cpp) — TEST INFRASTRUCTURE ONLY.

Only the test-suite, `__graft_entry__.smoke()` and the CPU leg of `bench.py` use this module,
as the checker / host-core baseline.  The renderer itself never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfhtgs_oracle.so")
_lock = threading.Lock()
_lib = None

u32p = C.POINTER(C.c_uint32)
u16p = C.POINTER(C.c_uint16)
u8p = C.POINTER(C.c_uint8)
f32p = C.POINTER(C.c_float)
i64p = C.POINTER(C.c_int64)


class OracleView(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int),
        ("focal_x", C.c_float), ("focal_y", C.c_float), ("center_x", C.c_float), ("center_y", C.c_float),
        ("near_plane", C.c_float), ("far_plane", C.c_float),
        ("M", C.c_float * 12), ("VPM", C.c_float * 16), ("VPR_inv", C.c_float * 16),
        ("cam_position", C.c_float * 3), ("gaze", C.c_float * 2),
        ("visibility_mask", u32p), ("visibility_mask_area_table", u32p), ("fovea_mask_area_table", u32p),
    ]


class OracleScene(C.Structure):
    _fields_ = [
        ("positions", f32p), ("scales", f32p), ("rotations", f32p), ("opacities", f32p),
        ("sh_0", f32p), ("sh_rest", f32p), ("n", C.c_int), ("total_sh_bases", C.c_int),
    ]


class OracleSettings(C.Structure):
    _fields_ = [
        ("K", C.c_int), ("active_sh_bases", C.c_int), ("scale_modifier", C.c_float),
        ("to_chw", C.c_int), ("blur_periphery", C.c_int), ("anti_aliasing", C.c_int),
        ("background_type", C.c_int), ("background_data", f32p),
        ("texture_width", C.c_int), ("texture_height", C.c_int),
        ("precision", C.c_int), ("n_threads", C.c_int),
        ("foveation", C.c_int), ("ring_full", C.c_float), ("ring_half", C.c_float),
    ]

FOVEATION = {"reference": 0, "rings": 1, "none": 2}


class OraclePrimitives(C.Structure):
    _fields_ = [("n_touched", u32p), ("screen_bounds", u16p), ("vpmt", f32p), ("rgba", f32p)]


class OracleTiles(C.Structure):
    _fields_ = [("tile_index_map_partitioned", u32p), ("tile_type_partitioned", u8p),
                ("partition_ranges", u32p), ("n_active_tiles", u32p)]


class OracleInstances(C.Structure):
    _fields_ = [("keys", u32p), ("values", u32p), ("capacity", C.c_int64), ("n_instances", i64p),
                ("instance_ranges", u32p)]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -fopenmp) if the library is missing."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(_LIB_PATH)
            L.oracle_view_geometry.argtypes = [C.POINTER(OracleView)] + [C.POINTER(C.c_int)] * 6
            L.oracle_classify_tiles.argtypes = [C.POINTER(OracleView), C.POINTER(OracleTiles)]
            L.oracle_preprocess.argtypes = [C.POINTER(OracleScene), C.POINTER(OracleView),
                                            C.POINTER(OracleSettings), C.POINTER(OraclePrimitives)]
            L.oracle_instances_from_primitives.argtypes = [C.POINTER(OracleView), C.c_int, u32p, u16p,
                                                           C.POINTER(OracleInstances), u32p, u32p]
            L.oracle_blend_compose.argtypes = [C.POINTER(OracleView), C.POINTER(OracleSettings), C.c_int,
                                               f32p, f32p, u32p, u32p, u32p, u32p, f32p]
            L.oracle_render_view.argtypes = [C.POINTER(OracleScene), C.POINTER(OracleView),
                                             C.POINTER(OracleSettings), f32p, C.POINTER(OraclePrimitives),
                                             C.POINTER(OracleTiles), C.POINTER(OracleInstances)]
            L.oracle_time_views.argtypes = [C.POINTER(OracleScene), C.POINTER(OracleView), C.c_int,
                                            C.POINTER(OracleSettings), C.POINTER(f32p)]
            L.oracle_time_views.restype = C.c_double
            L.oracle_stage_seconds.argtypes = [C.POINTER(C.c_double)]
            L.oracle_stage_seconds.restype = None
            _lib = L
    return _lib


def _p(a: np.ndarray, t):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(t)


class _Keep:
    """Holds numpy arrays alive while a ctypes struct points into them."""

    def __init__(self):
        self.refs = []

    def arr(self, a, dtype):
        a = np.ascontiguousarray(a, dtype)
        self.refs.append(a)
        return a


def make_view(v, keep: _Keep) -> OracleView:
    ov = OracleView()
    ov.width, ov.height = v.width, v.height
    ov.focal_x, ov.focal_y, ov.center_x, ov.center_y = v.focal_x, v.focal_y, v.center_x, v.center_y
    ov.near_plane, ov.far_plane = v.near_plane, v.far_plane
    ov.M[:] = [float(x) for x in np.asarray(v.M, np.float32).reshape(-1)]
    ov.VPM[:] = [float(x) for x in np.asarray(v.VPM, np.float32).reshape(-1)]
    ov.VPR_inv[:] = [float(x) for x in np.asarray(v.VPR_inv, np.float32).reshape(-1)]
    ov.cam_position[:] = [float(x) for x in np.asarray(v.cam_position, np.float32).reshape(-1)]
    ov.gaze[:] = [float(x) for x in np.asarray(v.gaze_position, np.float32).reshape(-1)]
    ov.visibility_mask = _p(keep.arr(v.visibility_mask, np.uint32), u32p)
    ov.visibility_mask_area_table = _p(keep.arr(v.visibility_mask_area_table, np.uint32), u32p)
    ov.fovea_mask_area_table = _p(keep.arr(v.fovea_mask_area_table, np.uint32), u32p)
    return ov


def make_scene(g, keep: _Keep) -> OracleScene:
    s = OracleScene()
    s.positions = _p(keep.arr(g.positions, np.float32), f32p)
    s.scales = _p(keep.arr(g.scales, np.float32), f32p)
    s.rotations = _p(keep.arr(g.rotations, np.float32), f32p)
    s.opacities = _p(keep.arr(g.opacities, np.float32), f32p)
    s.sh_0 = _p(keep.arr(g.sh_0, np.float32), f32p)
    rest = keep.arr(g.sh_rest if g.sh_rest.size else np.zeros((1,), np.float32), np.float32)
    s.sh_rest = _p(rest, f32p)
    s.n = g.n
    s.total_sh_bases = int(g.sh_rest.shape[1])
    return s


def make_settings(keep: _Keep, K=8, active_sh_bases=16, scale_modifier=1.0, to_chw=True, blur=False,
                  aaa=False, background=None, background_type=0, precision=64, n_threads=0,
                  foveation="reference", rings=(0.15, 0.4)) -> OracleSettings:
    st = OracleSettings()
    st.foveation = FOVEATION[foveation]
    st.ring_full, st.ring_half = float(rings[0]), float(rings[1])
    st.K, st.active_sh_bases, st.scale_modifier = K, active_sh_bases, scale_modifier
    st.to_chw, st.blur_periphery, st.anti_aliasing = int(to_chw), int(blur), int(aaa)
    st.background_type = background_type
    if background is None:
        background = np.zeros((1,), np.float32)
    bg = keep.arr(background, np.float32)
    st.background_data = _p(bg, f32p)
    if background_type in (2, 3):
        st.texture_width, st.texture_height = int(bg.shape[2]), int(bg.shape[1])
    st.precision, st.n_threads = precision, n_threads
    return st


def geometry(v) -> dict:
    keep = _Keep()
    ov = make_view(v, keep)
    vals = [C.c_int() for _ in range(6)]
    lib().oracle_view_geometry(C.byref(ov), *[C.byref(x) for x in vals])
    names = ["grid_large_w", "grid_large_h", "n_tiles", "end_bit", "gaze_tile_x", "gaze_tile_y"]
    return {k: x.value for k, x in zip(names, vals)}


def render(g, v, *, intermediates=False, **settings):
    """Render one view; returns the image ([3,H,W] or [H,W,3]) and optionally intermediates."""
    keep = _Keep()
    ov, sc = make_view(v, keep), make_scene(g, keep)
    st = make_settings(keep, **settings)
    shape = (3, v.height, v.width) if settings.get("to_chw", True) else (v.height, v.width, 3)
    img = np.zeros(shape, np.float32)
    if not intermediates:
        lib().oracle_render_view(C.byref(sc), C.byref(ov), C.byref(st), _p(img, f32p), None, None, None)
        return img
    geo = geometry(v)
    n, T = g.n, geo["n_tiles"]
    pr = dict(n_touched=np.zeros(n, np.uint32), screen_bounds=np.zeros((n, 4), np.uint16),
              vpmt=np.zeros((n, 12), np.float32), rgba=np.zeros((n, 4), np.float32))
    op = OraclePrimitives(_p(pr["n_touched"], u32p), _p(pr["screen_bounds"], u16p), _p(pr["vpmt"], f32p),
                          _p(pr["rgba"], f32p))
    tl = dict(tile_index_map_partitioned=np.zeros(T, np.uint32), tile_type_partitioned=np.zeros(T, np.uint8),
              partition_ranges=np.zeros(6, np.uint32), n_active_tiles=np.zeros(1, np.uint32))
    ot = OracleTiles(_p(tl["tile_index_map_partitioned"], u32p), _p(tl["tile_type_partitioned"], u8p),
                     _p(tl["partition_ranges"], u32p), _p(tl["n_active_tiles"], u32p))
    # instance capacity: sum of n_touched is only known after preprocess -> two calls
    lib().oracle_preprocess(C.byref(sc), C.byref(ov), C.byref(st), C.byref(op))
    m_cap = int(pr["n_touched"].astype(np.uint64).sum())
    inst = dict(keys=np.zeros(max(m_cap, 1), np.uint32), values=np.zeros(max(m_cap, 1), np.uint32),
                n_instances=np.zeros(1, np.int64), instance_ranges=np.zeros(2 * T, np.uint32))
    oi = OracleInstances(_p(inst["keys"], u32p), _p(inst["values"], u32p), m_cap, _p(inst["n_instances"], i64p),
                         _p(inst["instance_ranges"], u32p))
    lib().oracle_render_view(C.byref(sc), C.byref(ov), C.byref(st), _p(img, f32p), C.byref(op), C.byref(ot),
                             C.byref(oi))
    m = int(inst["n_instances"][0])
    out = dict(pr)
    na = int(tl["n_active_tiles"][0])
    out.update(tile_index_map_partitioned=tl["tile_index_map_partitioned"][:na],
               tile_type_partitioned=tl["tile_type_partitioned"][:na],
               partition_ranges=tl["partition_ranges"], n_active_tiles=na,
               keys=inst["keys"][:m], values=inst["values"][:m], n_instances=m,
               instance_ranges=inst["instance_ranges"].reshape(-1, 2), **geo)
    return img, out


def preprocess(g, v, **settings) -> dict:
    keep = _Keep()
    ov, sc = make_view(v, keep), make_scene(g, keep)
    st = make_settings(keep, **settings)
    n = g.n
    pr = dict(n_touched=np.zeros(n, np.uint32), screen_bounds=np.zeros((n, 4), np.uint16),
              vpmt=np.zeros((n, 12), np.float32), rgba=np.zeros((n, 4), np.float32))
    op = OraclePrimitives(_p(pr["n_touched"], u32p), _p(pr["screen_bounds"], u16p), _p(pr["vpmt"], f32p),
                          _p(pr["rgba"], f32p))
    lib().oracle_preprocess(C.byref(sc), C.byref(ov), C.byref(st), C.byref(op))
    return pr


def classify(v) -> dict:
    keep = _Keep()
    ov = make_view(v, keep)
    T = geometry(v)["n_tiles"]
    tl = dict(tile_index_map_partitioned=np.zeros(T, np.uint32), tile_type_partitioned=np.zeros(T, np.uint8),
              partition_ranges=np.zeros(6, np.uint32), n_active_tiles=np.zeros(1, np.uint32))
    ot = OracleTiles(_p(tl["tile_index_map_partitioned"], u32p), _p(tl["tile_type_partitioned"], u8p),
                     _p(tl["partition_ranges"], u32p), _p(tl["n_active_tiles"], u32p))
    lib().oracle_classify_tiles(C.byref(ov), C.byref(ot))
    na = int(tl["n_active_tiles"][0])
    return dict(tile_index_map_partitioned=tl["tile_index_map_partitioned"][:na],
                tile_type_partitioned=tl["tile_type_partitioned"][:na],
                partition_ranges=tl["partition_ranges"], n_active_tiles=na)


def instances(v, n_touched, screen_bounds) -> dict:
    """Instance creation + stable sort + ranges from given per-primitive counts/bounds."""
    keep = _Keep()
    ov = make_view(v, keep)
    T = geometry(v)["n_tiles"]
    nt = keep.arr(n_touched, np.uint32)
    sb = keep.arr(screen_bounds, np.uint16)
    m_cap = int(nt.astype(np.uint64).sum())
    out = dict(keys=np.zeros(max(m_cap, 1), np.uint32), values=np.zeros(max(m_cap, 1), np.uint32),
               n_instances=np.zeros(1, np.int64), instance_ranges=np.zeros(2 * T, np.uint32),
               keys_unsorted=np.zeros(max(m_cap, 1), np.uint32), values_unsorted=np.zeros(max(m_cap, 1), np.uint32))
    oi = OracleInstances(_p(out["keys"], u32p), _p(out["values"], u32p), m_cap, _p(out["n_instances"], i64p),
                         _p(out["instance_ranges"], u32p))
    lib().oracle_instances_from_primitives(C.byref(ov), int(nt.size), _p(nt, u32p), _p(sb, u16p), C.byref(oi),
                                           _p(out["keys_unsorted"], u32p), _p(out["values_unsorted"], u32p))
    m = int(out["n_instances"][0])
    for k in ("keys", "values", "keys_unsorted", "values_unsorted"):
        out[k] = out[k][:m]
    out["n_instances"] = m
    out["instance_ranges"] = out["instance_ranges"].reshape(-1, 2)
    return out


def blend_compose(v, n, vpmt, rgba, tile_index_map_partitioned, partition_ranges, sorted_values,
                  instance_ranges, **settings) -> np.ndarray:
    keep = _Keep()
    ov = make_view(v, keep)
    st = make_settings(keep, **settings)
    shape = (3, v.height, v.width) if settings.get("to_chw", True) else (v.height, v.width, 3)
    img = np.zeros(shape, np.float32)
    vp, rg = keep.arr(vpmt, np.float32), keep.arr(rgba, np.float32)
    tm = keep.arr(tile_index_map_partitioned if len(tile_index_map_partitioned) else np.zeros(1), np.uint32)
    prr = keep.arr(partition_ranges, np.uint32)
    sv = keep.arr(sorted_values if len(sorted_values) else np.zeros(1), np.uint32)
    ir = keep.arr(instance_ranges, np.uint32)
    lib().oracle_blend_compose(C.byref(ov), C.byref(st), int(n), _p(vp, f32p), _p(rg, f32p), _p(tm, u32p),
                               _p(prr, u32p), _p(sv, u32p), _p(ir, u32p), _p(img, f32p))
    return img


def time_views(g, views, n_threads=0, **settings) -> tuple[float, list]:
    """Renders `views` sequentially on the host cores; returns (seconds, images)."""
    keep = _Keep()
    sc = make_scene(g, keep)
    st = make_settings(keep, n_threads=n_threads, **settings)
    arr = (OracleView * len(views))(*[make_view(v, keep) for v in views])
    imgs = [np.zeros((3, v.height, v.width), np.float32) for v in views]
    ptrs = (f32p * len(views))(*[_p(i, f32p) for i in imgs])
    secs = lib().oracle_time_views(C.byref(sc), arr, len(views), C.byref(st), ptrs)
    return float(secs), imgs


def last_stage_seconds() -> dict:
    """Per-stage wall seconds of the last time_views call (std::chrono inside the oracle)."""
    out = (C.c_double * 4)()
    lib().oracle_stage_seconds(out)
    return dict(zip(("preprocess", "classify", "create_sort_ranges", "blend_compose"), [float(x) for x in out]))
