"""Access to the reference implementation built under oracle/_ref/ — TEST INFRASTRUCTURE ONLY.

* `intermediates(...)` runs the reference's own kernels through oracle/ref_harness.cu and
  returns every intermediate (per-primitive counts/bounds/VPMT/rgba, tile maps, sorted keys and
  values, tile ranges) for bit-exact comparison.
* `module(name)` imports the reference's pybind modules `_C`, `_C_benchmarking`, `_C_stereo`
  (built from its own sources by oracle/build_ref.sh) for end-to-end image comparison.
Only tests and fixture generation use this; nothing here is part of the renderer.
"""
from __future__ import annotations

import ctypes as C
import importlib
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_libs: dict[str, C.CDLL] = {}

vp = C.c_void_p
u32p = C.POINTER(C.c_uint32)
u16p = C.POINTER(C.c_uint16)
u8p = C.POINTER(C.c_uint8)
f32p = C.POINTER(C.c_float)
i64p = C.POINTER(C.c_int64)
i32p = C.POINTER(C.c_int32)


class RefArgs(C.Structure):
    _fields_ = [("positions", vp), ("scales", vp), ("rotations", vp), ("opacities", vp), ("sh_0", vp),
                ("sh_rest", vp), ("n", C.c_int), ("total_sh_bases", C.c_int), ("M", vp), ("VPM", vp),
                ("VPR_inv", vp), ("cam_position", vp), ("gaze_x", C.c_float), ("gaze_y", C.c_float),
                ("visibility_mask", vp), ("visibility_mask_area_table", vp), ("fovea_mask_area_table", vp),
                ("active_sh_bases", C.c_int), ("width", C.c_int), ("height", C.c_int), ("focal_x", C.c_float),
                ("focal_y", C.c_float), ("center_x", C.c_float), ("center_y", C.c_float),
                ("near_plane", C.c_float), ("far_plane", C.c_float), ("scale_modifier", C.c_float),
                ("anti_aliasing", C.c_int)]


class RefOut(C.Structure):
    _fields_ = [("n_touched", u32p), ("screen_bounds", u16p), ("vpmt", f32p), ("rgba", f32p), ("offsets", u32p),
                ("tile_index_map_partitioned", u32p), ("tile_type_partitioned", u8p), ("partition_ranges", u32p),
                ("n_active_tiles", u32p), ("keys_unsorted", u32p), ("values_unsorted", u32p), ("keys", u32p),
                ("values", u32p), ("capacity", C.c_int64), ("n_instances", i64p), ("instance_ranges", u32p),
                ("end_bit", i32p)]


def harness_path(fast: bool) -> str:
    return os.path.join(REF_DIR, "libref_harness_fast.so" if fast else "libref_harness_ieee.so")


def available() -> bool:
    return (os.path.exists(harness_path(True)) and os.path.exists(harness_path(False))
            and os.path.isdir(os.path.join(REF_DIR, "FoveatedHTGSCudaBackend")))


def _harness(fast: bool) -> C.CDLL:
    key = "fast" if fast else "ieee"
    if key not in _libs:
        lib = C.CDLL(harness_path(fast))
        lib.ref_intermediates.argtypes = [C.POINTER(RefArgs), C.POINTER(RefOut)]
        lib.ref_intermediates.restype = C.c_int
        _libs[key] = lib
    return _libs[key]


def module(name: str):
    """Imports the reference's extension module `name` from oracle/_ref (needs torch)."""
    import torch  # noqa: F401  (the modules link against libtorch)

    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    return importlib.import_module(f"FoveatedHTGSCudaBackend.{name}")


def intermediates(gaussians_t, settings, *, fast: bool = True, aaa: bool = False, capacity: int | None = None) -> dict:
    """Runs the reference's kernels for one view; tensors must be CUDA float32 / uint32(int32)."""
    import torch

    pos, scl, rot, opa, sh0, shr = [t.contiguous() for t in gaussians_t]
    n = int(pos.shape[0])
    s = settings
    a = RefArgs()
    a.positions, a.scales, a.rotations, a.opacities = pos.data_ptr(), scl.data_ptr(), rot.data_ptr(), opa.data_ptr()
    a.sh_0, a.sh_rest = sh0.data_ptr(), (shr.data_ptr() if shr.numel() else 0)
    a.n, a.total_sh_bases = n, int(shr.shape[1])
    keep = [t.contiguous() for t in (s.M, s.VPM, s.VPR_inv, s.cam_position, s.visibility_mask,
                                     s.visibility_mask_area_table, s.fovea_mask_area_table)]
    a.M, a.VPM, a.VPR_inv, a.cam_position = [t.data_ptr() for t in keep[:4]]
    g = s.gaze_position.reshape(-1).cpu()
    a.gaze_x, a.gaze_y = float(g[0]), float(g[1])
    a.visibility_mask, a.visibility_mask_area_table, a.fovea_mask_area_table = [t.data_ptr() for t in keep[4:]]
    a.active_sh_bases, a.width, a.height = int(s.active_sh_bases), int(s.width), int(s.height)
    a.focal_x, a.focal_y, a.center_x, a.center_y = float(s.focal_x), float(s.focal_y), float(s.center_x), float(s.center_y)
    a.near_plane, a.far_plane, a.scale_modifier = float(s.near_plane), float(s.far_plane), float(s.scale_modifier)
    a.anti_aliasing = int(aaa)
    W, H = int(s.width), int(s.height)
    T = 4 * ((W + 15) // 16) * ((H + 15) // 16)
    torch.cuda.synchronize()
    # capacity: upper bound from a first pass is not available; use the area tables' bound
    cap = capacity if capacity is not None else max(1, 64 * n + 1024)
    out = dict(n_touched=np.zeros(max(n, 1), np.uint32), screen_bounds=np.zeros((max(n, 1), 4), np.uint16),
               vpmt=np.zeros((max(n, 1), 12), np.float32), rgba=np.zeros((max(n, 1), 4), np.float32),
               offsets=np.zeros(max(n, 1), np.uint32), tile_index_map_partitioned=np.zeros(T, np.uint32),
               tile_type_partitioned=np.zeros(T, np.uint8), partition_ranges=np.zeros(6, np.uint32),
               n_active_tiles=np.zeros(1, np.uint32), keys_unsorted=np.zeros(cap, np.uint32),
               values_unsorted=np.zeros(cap, np.uint32), keys=np.zeros(cap, np.uint32),
               values=np.zeros(cap, np.uint32), n_instances=np.zeros(1, np.int64),
               instance_ranges=np.zeros((T, 2), np.uint32), end_bit=np.zeros(1, np.int32))

    def p(k, t):
        return out[k].ctypes.data_as(t)

    o = RefOut(p("n_touched", u32p), p("screen_bounds", u16p), p("vpmt", f32p), p("rgba", f32p), p("offsets", u32p),
               p("tile_index_map_partitioned", u32p), p("tile_type_partitioned", u8p), p("partition_ranges", u32p),
               p("n_active_tiles", u32p), p("keys_unsorted", u32p), p("values_unsorted", u32p), p("keys", u32p),
               p("values", u32p), cap, p("n_instances", i64p), p("instance_ranges", u32p), p("end_bit", i32p))
    rc = _harness(fast).ref_intermediates(C.byref(a), C.byref(o))
    if rc != 0:
        raise RuntimeError(f"reference harness failed with CUDA error {rc}")
    m = int(out["n_instances"][0])
    if m > cap:
        return intermediates(gaussians_t, settings, fast=fast, aaa=aaa, capacity=m)
    na = int(out["n_active_tiles"][0])
    for k in ("keys_unsorted", "values_unsorted", "keys", "values"):
        out[k] = out[k][:m]
    for k in ("n_touched", "screen_bounds", "vpmt", "rgba", "offsets"):
        out[k] = out[k][:n]
    out["tile_index_map_partitioned"] = out["tile_index_map_partitioned"][:na]
    out["tile_type_partitioned"] = out["tile_type_partitioned"][:na]
    out["n_instances"] = m
    out["n_active_tiles"] = na
    out["end_bit"] = int(out["end_bit"][0])
    return out
