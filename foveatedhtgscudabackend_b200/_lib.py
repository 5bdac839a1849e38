"""ctypes binding of libfhtgs.so (include/fhtgs.h).

The shared library is built in-tree by `foveatedhtgscudabackend_b200.build` (nvcc, sm_100a).
There is no fallback: if the library is missing or fails to load, every render call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libfhtgs.so")

c_f = C.c_float
c_i32 = C.c_int32
fp = C.POINTER(C.c_float)
u32p = C.POINTER(C.c_uint32)
u16p = C.POINTER(C.c_uint16)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p

N_STAGES = 7
WAIT_TEST_SORT_LOOKBACK = 1
WAIT_TEST_STAGING = 2
STAGE_NAMES = ["setup", "preprocess_classify", "scan_create", "sort", "ranges_order", "blend", "compose"]

STATUS = {
    0: "FHTGS_OK",
    1: "FHTGS_ERR_INVALID_ARGUMENT",
    2: "FHTGS_ERR_CUDA",
    3: "FHTGS_ERR_OUT_OF_MEMORY",
    4: "FHTGS_ERR_CAPACITY",
    5: "FHTGS_ERR_NOT_READY",
}


class FhtgsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Primitives(C.Structure):
    _fields_ = [("positions", vp), ("scales", vp), ("rotations", vp), ("opacities", vp), ("sh_0", vp),
                ("sh_rest", vp), ("n_primitives", c_i32), ("total_sh_bases", c_i32), ("storage", c_i32)]


STORAGE_FP32 = 0
STORAGE_HALF = 1


class View(C.Structure):
    _fields_ = [("M", vp), ("VPM", vp), ("VPR_inv", vp), ("cam_position", vp), ("gaze_x", c_f), ("gaze_y", c_f),
                ("visibility_mask", vp), ("visibility_mask_area_table", vp), ("fovea_mask_area_table", vp),
                ("width", c_i32), ("height", c_i32), ("focal_x", c_f), ("focal_y", c_f), ("center_x", c_f),
                ("center_y", c_f), ("image", vp), ("foveation", c_i32), ("ring_full", c_f), ("ring_half", c_f)]


class Settings(C.Structure):
    _fields_ = [("K", c_i32), ("active_sh_bases", c_i32), ("near_plane", c_f), ("far_plane", c_f),
                ("scale_modifier", c_f), ("to_chw", c_i32), ("blur_periphery", c_i32), ("anti_aliasing", c_i32),
                ("background_type", c_i32), ("background_data", vp), ("texture_width", c_i32),
                ("texture_height", c_i32), ("fast_math", c_i32), ("foveation", c_i32), ("ring_full", c_f),
                ("ring_half", c_f)]


FOVEATION = {"reference": 0, "rings": 1, "none": 2}


class FrameInfo(C.Structure):
    _fields_ = [("n_instances", C.c_int64), ("instance_capacity", C.c_int64), ("n_active_tiles", C.c_uint32),
                ("partition_ranges", C.c_uint32 * 6), ("overflow", c_i32), ("end_bit", c_i32),
                ("n_instances_stored", C.c_int64)]


class Intermediates(C.Structure):
    _fields_ = [("n_touched", u32p), ("screen_bounds", u16p), ("vpmt", fp), ("rgba", fp),
                ("tile_index_map_partitioned", u32p), ("tile_type_partitioned", u8p), ("keys", u32p),
                ("values", u32p), ("instance_ranges", u32p)]


class Tuning(C.Structure):
    _fields_ = [("blend_warp_width", c_i32), ("blend_blocks_per_sm", c_i32), ("sort_items", c_i32)]


class ServerConfig(C.Structure):
    _fields_ = [("device", c_i32), ("max_in_flight", c_i32), ("max_batch_requests", c_i32),
                ("blend_split_permille", c_i32),
                ("hbm_budget_bytes", C.c_int64)]


class Eye(C.Structure):
    _fields_ = [("M", c_f * 12), ("VPM", c_f * 16), ("VPR_inv", c_f * 16), ("cam_position", c_f * 3),
                ("gaze_x", c_f), ("gaze_y", c_f), ("width", c_i32), ("height", c_i32), ("focal_x", c_f),
                ("focal_y", c_f), ("center_x", c_f), ("center_y", c_f), ("visibility_mask", vp),
                ("visibility_mask_area_table", vp), ("fovea_mask_area_table", vp), ("image", vp)]


class Request(C.Structure):
    _fields_ = [("scene", c_i32), ("n_eyes", c_i32), ("tag", C.c_uint64), ("ready_event", vp), ("eyes", Eye * 2)]


class Completion(C.Structure):
    _fields_ = [("ticket", C.c_int64), ("tag", C.c_uint64), ("status", c_i32), ("frame_views", c_i32),
                ("submit_ms", C.c_double), ("launch_ms", C.c_double), ("done_ms", C.c_double),
                ("images", vp * 2), ("message", C.c_char * 96)]


class GroupCompletion(C.Structure):
    _fields_ = [("completion", Completion), ("replica", c_i32), ("device", c_i32)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("submitted", "completed", "failed", "frames", "views", "retries", "queued",
                                         "in_flight", "resident_bytes", "peak_resident_bytes", "admission_waits",
                                         "max_frame_requests")]


# Exported symbols and their signatures (mirrors include/fhtgs.h).
_MONO_ARGS = [vp, vp, vp, vp, vp, vp, vp, c_i32, c_i32, vp, vp, vp, vp, c_f, c_f, vp, vp, vp, vp, c_i32, c_i32,
              c_i32, c_i32, c_i32, c_i32, c_i32, c_f, c_f, c_f, c_f, c_f, c_f, c_f, c_i32, c_i32, c_i32, vp, vp]
_STEREO_ARGS = ([vp, vp, vp, vp, vp, vp, vp, c_i32, c_i32]
                + [vp, vp, vp, vp, c_f, c_f, vp, vp, vp, vp, c_i32, c_i32, c_i32, c_i32, c_i32, c_i32, c_i32,
                   c_f, c_f, c_f, c_f, c_f, c_f, c_f]
                + [vp, vp, vp, vp, c_f, c_f, vp, vp, vp, c_i32, c_i32, c_f, c_f, c_f, c_f]
                + [c_i32, c_i32, c_i32, vp, vp, vp])
SIGNATURES = {
    "fhtgs_abi_version": ([], c_i32),
    "fhtgs_last_error": ([], C.c_char_p),
    "fhtgs_context_create": ([c_i32, C.POINTER(vp)], c_i32),
    "fhtgs_context_destroy": ([vp], c_i32),
    "fhtgs_context_reserve": ([vp, c_i32, c_i32, c_i32, c_i32, C.c_int64], c_i32),
    "fhtgs_context_arena_bytes": ([vp], C.c_size_t),
    "fhtgs_context_launch_count": ([vp], C.c_int64),
    "fhtgs_context_set_profiling": ([vp, c_i32], c_i32),
    "fhtgs_get_stage_times": ([vp, C.POINTER(C.c_float), c_i32], c_i32),
    "fhtgs_get_stage_history": ([vp, C.POINTER(C.c_float), c_i32, C.POINTER(c_i32)], c_i32),
    "fhtgs_render_views": ([vp, C.POINTER(Primitives), C.POINTER(View), c_i32, C.POINTER(Settings), vp], c_i32),
    "fhtgs_render_views_sync": ([vp, C.POINTER(Primitives), C.POINTER(View), c_i32, C.POINTER(Settings), vp], c_i32),
    "fhtgs_get_frame_info": ([vp, c_i32, C.POINTER(FrameInfo)], c_i32),
    "fhtgs_copy_intermediates": ([vp, c_i32, C.POINTER(Intermediates)], c_i32),
    "fhtgs_context_test_wait_timeout": ([vp, c_i32, c_i32], c_i32),
    "fhtgs_render_mono": (_MONO_ARGS, c_i32),
    "fhtgs_benchmark_mono": (_MONO_ARGS, c_i32),
    "fhtgs_render_stereo": (_STEREO_ARGS, c_i32),
    "fhtgs_sort_instances_noalloc": ([vp, vp, vp, vp, C.c_int64, c_i32, c_i32, vp], c_i32),
    "fhtgs_context_set_tuning": ([vp, C.POINTER(Tuning)], c_i32),
    "fhtgs_context_get_tuning": ([vp, C.POINTER(Tuning)], c_i32),
    "fhtgs_context_set_blend_split": ([vp, c_f, c_i32], c_i32),
    "fhtgs_context_set_blend_split_exact": ([vp, c_i32, C.c_int64], c_i32),
    "fhtgs_context_get_blend_split_stats": ([vp] + [C.POINTER(c_i32)] * 4, c_i32),
    "fhtgs_autotune": ([vp, C.POINTER(Primitives), C.POINTER(View), c_i32, C.POINTER(Settings), c_i32,
                        C.POINTER(Tuning), C.POINTER(C.c_float), vp], c_i32),
    "fhtgs_frame_graph_create": ([vp, C.POINTER(Primitives), C.POINTER(View), c_i32, C.POINTER(Settings), vp, c_f,
                                  C.POINTER(vp), vp], c_i32),
    "fhtgs_frame_graph_launch": ([vp, vp], c_i32),
    "fhtgs_frame_graph_destroy": ([vp], c_i32),
    "fhtgs_server_create": ([C.POINTER(ServerConfig), C.POINTER(vp)], c_i32),
    "fhtgs_server_destroy": ([vp], c_i32),
    "fhtgs_server_add_scene": ([vp, C.POINTER(Primitives), C.POINTER(Settings), C.POINTER(c_i32)], c_i32),
    "fhtgs_server_remove_scene": ([vp, c_i32], c_i32),
    "fhtgs_server_submit": ([vp, C.POINTER(Request), C.POINTER(C.c_int64)], c_i32),
    "fhtgs_server_poll": ([vp, C.POINTER(Completion), c_i32, c_i32, C.POINTER(c_i32)], c_i32),
    "fhtgs_server_release": ([vp, C.c_int64], c_i32),
    "fhtgs_server_set_paused": ([vp, c_i32], c_i32),
    "fhtgs_server_drain": ([vp, c_i32], c_i32),
    "fhtgs_server_get_stats": ([vp, C.POINTER(ServerStats)], c_i32),
    "fhtgs_server_clock_ms": ([vp], C.c_double),
    "fhtgs_server_group_create": ([C.POINTER(c_i32), c_i32, C.POINTER(ServerConfig), C.POINTER(vp)], c_i32),
    "fhtgs_server_group_destroy": ([vp], c_i32),
    "fhtgs_server_group_size": ([vp], c_i32),
    "fhtgs_server_group_add_scene": ([vp, c_i32, C.POINTER(Primitives), C.POINTER(Settings), C.POINTER(c_i32)], c_i32),
    "fhtgs_server_group_remove_scene": ([vp, c_i32], c_i32),
    "fhtgs_server_group_submit": ([vp, C.POINTER(Request), C.POINTER(C.c_int64), C.POINTER(c_i32)], c_i32),
    "fhtgs_server_group_poll": ([vp, C.POINTER(GroupCompletion), c_i32, c_i32, C.POINTER(c_i32)], c_i32),
    "fhtgs_server_group_release": ([vp, C.c_int64], c_i32),
    "fhtgs_server_group_drain": ([vp, c_i32], c_i32),
    "fhtgs_server_group_get_stats": ([vp, c_i32, C.POINTER(ServerStats), C.POINTER(C.c_int64)], c_i32),
    "fhtgs_build_tile_masks": ([vp, c_i32, c_i32, vp, vp, vp, vp], c_i32),
    "fhtgs_pack_display": ([C.POINTER(vp), c_i32, c_i32, c_i32, c_i32, c_i32, vp, vp], c_i32),
    "fhtgs_visualize_gaze": ([vp, c_i32, c_i32, c_f, c_f, c_f, c_f, c_f, c_i32, c_i32, c_i32, vp], c_i32),
    "fhtgs_visualize_tile_boundaries": ([vp, c_i32, c_i32, vp, c_f, c_f, c_i32, vp], c_i32),
}

_lock = threading.Lock()
_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Loads libfhtgs.so and declares every entry point; raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise FhtgsError(2, f"{p} is missing; build it with `python -m foveatedhtgscudabackend_b200.build`")
        lib = C.CDLL(p)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        if path is None:
            _lib = lib
        return lib


def check(status: int) -> None:
    if status != 0:
        msg = load().fhtgs_last_error()
        raise FhtgsError(status, msg.decode() if msg else "")


_contexts: dict[int, int] = {}


def context(device: int) -> int:
    """Process-wide context per CUDA device (owns the device arena)."""
    with _lock:
        h = _contexts.get(device)
    if h is None:
        out = vp()
        check(load().fhtgs_context_create(device, C.byref(out)))
        with _lock:
            _contexts[device] = out.value
            h = out.value
    return h
