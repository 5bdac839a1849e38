"""Drop-in Python surface of the reference's rasterization path.

Mirrors `FoveatedHTGSCudaBackend/torch_bindings/rasterization.py` of the reference:
`BackgroundModel` (:9-13), `RasterizerSettings` (:22-68, same field order and `as_tuple`),
`FoveatedHTGSRasterizer.render / benchmark / render_stereo` (:73-154), and the positional
extension entry points `_C.render` (30 args), `_C_benchmarking.benchmark` (30) and
`_C_stereo.render` (51) of `torch_bindings/bindings*.cpp`.  Every call goes through the C ABI
of libfhtgs.so (include/fhtgs.h); PyTorch only provides the tensors and the stream.

Differences from the reference, by design: inputs are made contiguous and kept alive for the
call; invalid inputs raise `FhtgsError` instead of running into undefined behaviour; the
render runs on PyTorch's current stream and the call returns when the images are complete
(the reference also blocks, on its private streams).
"""
from __future__ import annotations

import ctypes as C
from enum import Enum
from typing import NamedTuple

import torch

from . import _lib


class BackgroundModel(Enum):
    NONE = 0
    SH = 1
    TEXTURE = 2
    TEXTURE_RAW = 3  # texture storing pre-activation values, activated after interpolation


class GazeVisualizationType(Enum):
    CIRCLE = 0
    SQUARE = 1
    CROSS = 2


class RasterizerSettings(NamedTuple):
    M: torch.Tensor  # affine transformation from world space to view space [3,4]
    VPM: torch.Tensor  # homogeneous transformation from world space to screen space [4,4]
    VPR_inv: torch.Tensor  # screen space -> world direction, translation ignored [4,4]
    cam_position: torch.Tensor  # camera position in world space [3]
    gaze_position: torch.Tensor  # gaze position in screen space [2] (pixels)
    visibility_mask: torch.Tensor  # bit per 16x16 tile, uint32 words
    visibility_mask_area_table: torch.Tensor  # summed-area table of the mask, (gx+1)*(gy+1)
    fovea_mask_area_table: torch.Tensor  # 49x49 summed-area table of the fovea shape
    background_model_data: torch.Tensor  # background model specific data
    background_model: BackgroundModel
    K: int  # size of the core for hybrid transparency
    active_sh_bases: int  # number of spherical harmonics bases used for colour
    width: int
    height: int
    focal_x: float
    focal_y: float
    center_x: float
    center_y: float
    near_plane: float
    far_plane: float
    scale_modifier: float  # scaling factor applied to each Gaussian

    def as_tuple(self) -> tuple:
        return (
            self.M, self.VPM, self.VPR_inv, self.cam_position, self.gaze_position, self.visibility_mask,
            self.visibility_mask_area_table, self.fovea_mask_area_table, self.background_model_data,
            self.background_model.value, self.K, self.active_sh_bases, self.width, self.height, self.focal_x,
            self.focal_y, self.center_x, self.center_y, self.near_plane, self.far_plane, self.scale_modifier,
        )


# ---------------------------------------------------------------------------------------------
# tensor plumbing
# ---------------------------------------------------------------------------------------------
class _Keep:
    """Keeps the contiguous copies of the inputs alive until the render call returned."""

    def __init__(self, device: torch.device):
        self.device = device
        self.refs: list[torch.Tensor] = []

    def f32(self, t: torch.Tensor, name: str) -> int:
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor")
        if t.device != self.device:
            raise ValueError(f"{name} must be on {self.device}, got {t.device}")
        if t.dtype != torch.float32:
            raise TypeError(f"{name} must be float32, got {t.dtype}")
        t = t.contiguous()
        self.refs.append(t)
        return t.data_ptr() if t.numel() else 0

    def typed(self, t: torch.Tensor, name: str, dtype: torch.dtype) -> int:
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor")
        if t.device != self.device:
            raise ValueError(f"{name} must be on {self.device}, got {t.device}")
        if t.dtype != dtype:
            raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
        t = t.contiguous()
        self.refs.append(t)
        return t.data_ptr() if t.numel() else 0

    def u32(self, t: torch.Tensor, name: str) -> int:
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor")
        if t.device != self.device:
            raise ValueError(f"{name} must be on {self.device}, got {t.device}")
        if t.dtype not in (torch.int32, torch.uint32):
            raise TypeError(f"{name} must be uint32 (or int32 bit pattern), got {t.dtype}")
        t = t.contiguous()
        self.refs.append(t)
        return t.data_ptr()


def _gaze_xy(g: torch.Tensor) -> tuple[float, float]:
    g = g.detach().reshape(-1)
    if g.numel() < 2:
        raise ValueError("gaze_position needs two values")
    g = g[:2].to("cpu", torch.float32)
    return float(g[0]), float(g[1])


def _texture_size(bg_type: int, data: torch.Tensor) -> tuple[int, int]:
    if bg_type in (2, 3):
        if data.dim() != 3 or data.shape[0] != 3:
            raise ValueError("texture background data must be [3, h, w]")
        return int(data.shape[2]), int(data.shape[1])
    return 0, 0


def _check_gaussians(positions, scales, rotations, opacities, sh_0, sh_rest):
    if positions.dim() != 2 or positions.shape[1] != 3:
        raise ValueError("positions must be [N,3]")
    n = positions.shape[0]
    for name, t, w in (("scales", scales, 3), ("rotations", rotations, 4)):
        if t.shape[0] != n or t.numel() != n * w:
            raise ValueError(f"{name} must be [N,{w}]")
    if opacities.numel() != n:
        raise ValueError("opacities must hold N values")
    if sh_0.numel() != 3 * n:
        raise ValueError("sh_0 must be [N,1,3] or [N,3]")
    if sh_rest.shape[0] != n or (sh_rest.numel() and sh_rest.shape[-1] != 3):
        raise ValueError("sh_rest must be [N,S,3]")
    return n, int(sh_rest.shape[1]) if sh_rest.dim() >= 2 else 0


def _alloc_image(to_chw: bool, h: int, w: int, device) -> torch.Tensor:
    shape = (3, h, w) if to_chw else (h, w, 3)
    return torch.empty(shape, dtype=torch.float32, device=device)


def _stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _mono(fast: bool, positions, scales, rotations, opacities, sh_0, sh_rest, M, VPM, VPR_inv, cam_position,
          gaze_position, visibility_mask, visibility_mask_area_table, fovea_mask_area_table, background_model_data,
          background_model_type, K, active_sh_bases, width, height, focal_x, focal_y, center_x, center_y,
          near_plane, far_plane, scale_modifier, to_chw, blur_periphery, anti_aliasing) -> torch.Tensor:
    dev = positions.device
    if dev.type != "cuda":
        raise ValueError("positions must be a CUDA tensor")
    keep = _Keep(dev)
    n, total_sh = _check_gaussians(positions, scales, rotations, opacities, sh_0, sh_rest)
    gx, gy = _gaze_xy(gaze_position)
    bg_type = int(background_model_type)
    tw, th = _texture_size(bg_type, background_model_data)
    image = _alloc_image(bool(to_chw), int(height), int(width), dev)
    lib = _lib.load()
    fn = lib.fhtgs_benchmark_mono if fast else lib.fhtgs_render_mono
    with torch.cuda.device(dev):
        ctx = _lib.context(dev.index if dev.index is not None else torch.cuda.current_device())
        st = fn(ctx, keep.f32(positions, "positions"), keep.f32(scales, "scales"), keep.f32(rotations, "rotations"),
                keep.f32(opacities, "opacities"), keep.f32(sh_0, "sh_0"), keep.f32(sh_rest, "sh_rest"), n, total_sh,
                keep.f32(M, "M"), keep.f32(VPM, "VPM"), keep.f32(VPR_inv, "VPR_inv"),
                keep.f32(cam_position, "cam_position"), gx, gy, keep.u32(visibility_mask, "visibility_mask"),
                keep.u32(visibility_mask_area_table, "visibility_mask_area_table"),
                keep.u32(fovea_mask_area_table, "fovea_mask_area_table"),
                keep.f32(background_model_data, "background_model_data"), tw, th, bg_type, int(K),
                int(active_sh_bases), int(width), int(height), float(focal_x), float(focal_y), float(center_x),
                float(center_y), float(near_plane), float(far_plane), float(scale_modifier), int(bool(to_chw)),
                int(bool(blur_periphery)), int(bool(anti_aliasing)), image.data_ptr(), _stream_handle(dev))
    _lib.check(st)
    return image


class _CModule:
    """Stand-in for the reference's `_C` extension module: `render(*30 positional args)`."""

    @staticmethod
    def render(*args) -> torch.Tensor:
        if len(args) != 30:
            raise TypeError(f"render() takes 30 positional arguments ({len(args)} given)")
        return _mono(False, *args)


class _CBenchmarkingModule:
    """Stand-in for `_C_benchmarking`: `benchmark(*30 positional args)` (fast-math arithmetic)."""

    @staticmethod
    def benchmark(*args) -> torch.Tensor:
        if len(args) != 30:
            raise TypeError(f"benchmark() takes 30 positional arguments ({len(args)} given)")
        return _mono(True, *args)


class _CStereoModule:
    """Stand-in for `_C_stereo`: `render(*51 positional args)` -> (left, right)."""

    @staticmethod
    def render(*args) -> tuple[torch.Tensor, torch.Tensor]:
        if len(args) != 51:
            raise TypeError(f"render() takes 51 positional arguments ({len(args)} given)")
        g = args[:6]
        L = args[6:27]
        R = args[27:48]
        to_chw, blur_periphery, anti_aliasing = args[48:51]
        positions, scales, rotations, opacities, sh_0, sh_rest = g
        dev = positions.device
        if dev.type != "cuda":
            raise ValueError("positions must be a CUDA tensor")
        keep = _Keep(dev)
        n, total_sh = _check_gaussians(*g)
        (M_l, VPM_l, VPRi_l, cam_l, gaze_l, vis_l, vsat_l, fsat_l, bg_l, bgt_l, K_l, ash_l, w_l, h_l, fx_l, fy_l,
         cx_l, cy_l, near_l, far_l, sm_l) = L
        (M_r, VPM_r, VPRi_r, cam_r, gaze_r, vis_r, vsat_r, fsat_r, _bg_r, _bgt_r, _K_r, _ash_r, w_r, h_r, fx_r, fy_r,
         cx_r, cy_r, _near_r, _far_r, _sm_r) = R
        glx, gly = _gaze_xy(gaze_l)
        grx, gry = _gaze_xy(gaze_r)
        bg_type = int(bgt_l)
        tw, th = _texture_size(bg_type, bg_l)
        img_l = _alloc_image(bool(to_chw), int(h_l), int(w_l), dev)
        img_r = _alloc_image(bool(to_chw), int(h_r), int(w_r), dev)
        lib = _lib.load()
        with torch.cuda.device(dev):
            ctx = _lib.context(dev.index if dev.index is not None else torch.cuda.current_device())
            st = lib.fhtgs_render_stereo(
                ctx, keep.f32(positions, "positions"), keep.f32(scales, "scales"), keep.f32(rotations, "rotations"),
                keep.f32(opacities, "opacities"), keep.f32(sh_0, "sh_0"), keep.f32(sh_rest, "sh_rest"), n, total_sh,
                keep.f32(M_l, "M_left"), keep.f32(VPM_l, "VPM_left"), keep.f32(VPRi_l, "VPR_inv_left"),
                keep.f32(cam_l, "cam_position_left"), glx, gly, keep.u32(vis_l, "visibility_mask_left"),
                keep.u32(vsat_l, "visibility_mask_area_table_left"), keep.u32(fsat_l, "fovea_mask_area_table_left"),
                keep.f32(bg_l, "background_model_data_left"), tw, th, bg_type, int(K_l), int(ash_l), int(w_l),
                int(h_l), float(fx_l), float(fy_l), float(cx_l), float(cy_l), float(near_l), float(far_l),
                float(sm_l),
                keep.f32(M_r, "M_right"), keep.f32(VPM_r, "VPM_right"), keep.f32(VPRi_r, "VPR_inv_right"),
                keep.f32(cam_r, "cam_position_right"), grx, gry, keep.u32(vis_r, "visibility_mask_right"),
                keep.u32(vsat_r, "visibility_mask_area_table_right"), keep.u32(fsat_r, "fovea_mask_area_table_right"),
                int(w_r), int(h_r), float(fx_r), float(fy_r), float(cx_r), float(cy_r),
                int(bool(to_chw)), int(bool(blur_periphery)), int(bool(anti_aliasing)),
                img_l.data_ptr(), img_r.data_ptr(), _stream_handle(dev))
        _lib.check(st)
        return img_l, img_r


_C = _CModule()
_C_benchmarking = _CBenchmarkingModule()
_C_stereo = _CStereoModule()


class FoveatedHTGSRasterizer(torch.nn.Module):
    """Same methods and arguments as the reference's FoveatedHTGSRasterizer."""

    def render(self, positions, scales, rotations, opacities, sh_0, sh_rest, settings: RasterizerSettings,
               to_chw: bool, blur_periphery: bool, aaa_mode: bool) -> torch.Tensor:
        return _C.render(positions, scales, rotations, opacities, sh_0, sh_rest, *settings.as_tuple(), to_chw,
                         blur_periphery, aaa_mode)

    def benchmark(self, positions, scales, rotations, opacities, sh_0, sh_rest, settings: RasterizerSettings,
                  to_chw: bool, blur_periphery: bool, aaa_mode: bool) -> torch.Tensor:
        return _C_benchmarking.benchmark(positions, scales, rotations, opacities, sh_0, sh_rest,
                                         *settings.as_tuple(), to_chw, blur_periphery, aaa_mode)

    def render_stereo(self, positions, scales, rotations, opacities, sh_0, sh_rest,
                      settings_left: RasterizerSettings, settings_right: RasterizerSettings, to_chw: bool,
                      blur_periphery: bool, aaa_mode: bool) -> tuple[torch.Tensor, torch.Tensor]:
        return _C_stereo.render(positions, scales, rotations, opacities, sh_0, sh_rest, *settings_left.as_tuple(),
                                *settings_right.as_tuple(), to_chw, blur_periphery, aaa_mode)


# ---------------------------------------------------------------------------------------------
# multi-view interface (n views of one scene in one frame) + parity inspection
# ---------------------------------------------------------------------------------------------
class Renderer:
    """Owns a libfhtgs context; renders any number of views of one scene per call."""

    def __init__(self, device: int | torch.device | None = None):
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        if dev.type != "cuda":
            dev = torch.device("cuda", dev.index or 0)
        self.device = dev
        self._libh = _lib.load()
        out = _lib.vp()
        with torch.cuda.device(dev):
            _lib.check(self._libh.fhtgs_context_create(dev.index or 0, C.byref(out)))
        self.ctx = out.value
        self._last_views = 0
        self._last_n = 0
        self._foveation = (0, 0.0, 0.0)

    def close(self):
        if getattr(self, "ctx", None):
            self._libh.fhtgs_context_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_foveation(self, mode: str = "reference", ring_full: float = 0.15, ring_half: float = 0.4):
        """Foveation of this renderer's frames (fhtgs_settings.foveation): "reference" (the
        reference's fixed fovea / blend band / 2x periphery, the default), "rings" (full
        resolution within NDC radius ring_full of the gaze, 2x down within ring_half, 4x down
        beyond) or "none" (every tile at full resolution)."""
        if mode not in _lib.FOVEATION:
            raise ValueError(f"foveation must be one of {sorted(_lib.FOVEATION)}")
        self._foveation = (_lib.FOVEATION[mode], float(ring_full), float(ring_half))

    def reserve(self, n_primitives: int, n_views: int, max_width: int, max_height: int, instances_per_view: int = 0):
        _lib.check(self._libh.fhtgs_context_reserve(self.ctx, n_primitives, n_views, max_width, max_height,
                                                    int(instances_per_view)))

    def arena_bytes(self) -> int:
        return int(self._libh.fhtgs_context_arena_bytes(self.ctx))

    def launch_count(self) -> int:
        """Kernels this renderer's context has launched so far."""
        return int(self._libh.fhtgs_context_launch_count(self.ctx))

    def set_profiling(self, enable: bool = True):
        """Records CUDA events between the pipeline stages of every frame."""
        _lib.check(self._libh.fhtgs_context_set_profiling(self.ctx, int(bool(enable))))

    def stage_times(self) -> dict:
        """Milliseconds per stage of the last frame (waits for it)."""
        buf = (C.c_float * _lib.N_STAGES)()
        _lib.check(self._libh.fhtgs_get_stage_times(self.ctx, buf, _lib.N_STAGES))
        return dict(zip(_lib.STAGE_NAMES, [float(x) for x in buf]))

    def stage_history(self, max_frames: int = 64) -> list[dict]:
        """Stage milliseconds of up to the last 64 profiled frames, oldest first."""
        buf = (C.c_float * (_lib.N_STAGES * max_frames))()
        n = C.c_int32(0)
        _lib.check(self._libh.fhtgs_get_stage_history(self.ctx, buf, max_frames, C.byref(n)))
        return [dict(zip(_lib.STAGE_NAMES, [float(x) for x in buf[f * _lib.N_STAGES:(f + 1) * _lib.N_STAGES]]))
                for f in range(n.value)]

    def _frame(self, positions, scales, rotations, opacities, sh_0, sh_rest, settings, to_chw, blur_periphery,
               aaa_mode, fast_math, images, view_foveation=None):
        """C structures of one frame: (keep-alive, primitives, views array, settings, images)."""
        dev = self.device
        keep = _Keep(dev)
        n, total_sh = _check_gaussians(positions, scales, rotations, opacities, sh_0, sh_rest)
        if isinstance(scales, torch.Tensor) and scales.dtype == torch.float16:
            # reduced-precision storage: fp16 scales/rotations/opacities, bf16 SH, fp32 positions
            h, b = torch.float16, torch.bfloat16
            prims = _lib.Primitives(keep.f32(positions, "positions"), keep.typed(scales, "scales", h),
                                    keep.typed(rotations, "rotations", h), keep.typed(opacities, "opacities", h),
                                    keep.typed(sh_0, "sh_0", b), keep.typed(sh_rest, "sh_rest", b), n, total_sh,
                                    _lib.STORAGE_HALF)
        else:
            prims = _lib.Primitives(keep.f32(positions, "positions"), keep.f32(scales, "scales"),
                                    keep.f32(rotations, "rotations"), keep.f32(opacities, "opacities"),
                                    keep.f32(sh_0, "sh_0"), keep.f32(sh_rest, "sh_rest"), n, total_sh,
                                    _lib.STORAGE_FP32)
        s0 = settings[0]
        bg_type = s0.background_model.value
        tw, th = _texture_size(bg_type, s0.background_model_data)
        st = _lib.Settings(int(s0.K), int(s0.active_sh_bases), float(s0.near_plane), float(s0.far_plane),
                           float(s0.scale_modifier), int(bool(to_chw)), int(bool(blur_periphery)), int(bool(aaa_mode)),
                           bg_type, keep.f32(s0.background_model_data, "background_model_data"), tw, th,
                           int(bool(fast_math)), *self._foveation)
        if images is None:
            images = [_alloc_image(to_chw, int(s.height), int(s.width), dev) for s in settings]
        views = (_lib.View * len(settings))()
        for i, s in enumerate(settings):
            gx, gy = _gaze_xy(s.gaze_position)
            views[i] = _lib.View(keep.f32(s.M, "M"), keep.f32(s.VPM, "VPM"), keep.f32(s.VPR_inv, "VPR_inv"),
                                 keep.f32(s.cam_position, "cam_position"), gx, gy,
                                 keep.u32(s.visibility_mask, "visibility_mask"),
                                 keep.u32(s.visibility_mask_area_table, "visibility_mask_area_table"),
                                 keep.u32(s.fovea_mask_area_table, "fovea_mask_area_table"), int(s.width),
                                 int(s.height), float(s.focal_x), float(s.focal_y), float(s.center_x),
                                 float(s.center_y), images[i].data_ptr())
            if view_foveation is not None and view_foveation[i] is not None:
                mode, *radii = view_foveation[i] if isinstance(view_foveation[i], (tuple, list)) else (view_foveation[i],)
                if mode not in _lib.FOVEATION:
                    raise ValueError(f"foveation must be one of {sorted(_lib.FOVEATION)}")
                rf, rh = (list(radii) + [0.15, 0.4][len(radii):])[:2]
                views[i].foveation = _lib.FOVEATION[mode] + 1
                views[i].ring_full, views[i].ring_half = float(rf), float(rh)
        return keep, prims, views, st, images, n

    def render(self, positions, scales, rotations, opacities, sh_0, sh_rest, settings: list[RasterizerSettings],
               to_chw: bool = True, blur_periphery: bool = False, aaa_mode: bool = False, fast_math: bool = True,
               images: list[torch.Tensor] | None = None, sync: bool = True,
               view_foveation: list | None = None) -> list[torch.Tensor]:
        """Renders len(settings) views; K, SH bases, planes, scale and background of settings[0] apply.
        `view_foveation[i]` (optional): view i's own foveation, "reference" / "none" or
        ("rings", ring_full, ring_half), instead of the renderer's (set_foveation)."""
        dev = self.device
        keep, prims, views, st, images, n = self._frame(positions, scales, rotations, opacities, sh_0, sh_rest,
                                                        settings, to_chw, blur_periphery, aaa_mode, fast_math, images,
                                                        view_foveation)
        fn = self._libh.fhtgs_render_views_sync if sync else self._libh.fhtgs_render_views
        with torch.cuda.device(dev):
            _lib.check(fn(self.ctx, C.byref(prims), views, len(settings), C.byref(st), _stream_handle(dev)))
        if not sync:
            self._keep_async = keep  # inputs must outlive the queued frame
        self._last_views = len(settings)
        self._last_n = n
        self._last_sizes = [(int(s.width), int(s.height)) for s in settings]
        return images

    # ---- batched frames: tuning, autotuner, captured frame graphs ----

    def get_tuning(self) -> dict:
        t = _lib.Tuning()
        _lib.check(self._libh.fhtgs_context_get_tuning(self.ctx, C.byref(t)))
        return dict(blend_warp_width=int(t.blend_warp_width), blend_blocks_per_sm=int(t.blend_blocks_per_sm),
                    sort_items=int(t.sort_items))

    def set_tuning(self, blend_warp_width: int = 8, blend_blocks_per_sm: int = 0, sort_items: int = 16):
        """Kernel shapes of this context (identical images for every choice)."""
        t = _lib.Tuning(int(blend_warp_width), int(blend_blocks_per_sm), int(sort_items))
        _lib.check(self._libh.fhtgs_context_set_tuning(self.ctx, C.byref(t)))

    def set_blend_split(self, segment_share: float = 0.0, records: int = 0, exact: bool = False,
                        log_bytes: int = 0):
        """Split blend (0 = off, the default): full-resolution tiles whose list exceeds
        segment_share x (instances / blend blocks) are blended as segments on several blocks.
        exact=False: merged exactly up to the tail's summation order (fhtgs_context_set_blend_split);
        exact=True: the segments log their fragments and the merge replays them in order, images
        bit-identical to the default path (fhtgs_context_set_blend_split_exact)."""
        _lib.check(self._libh.fhtgs_context_set_blend_split(self.ctx, float(segment_share), int(records)))
        _lib.check(self._libh.fhtgs_context_set_blend_split_exact(self.ctx, 1 if exact else 0, int(log_bytes)))

    def blend_split_stats(self) -> dict:
        """The last frame's split blend: tiles split, segments, tiles blended whole after a record
        overflow, and the most records one pixel of a segment produced."""
        t, g, f, m = C.c_int32(0), C.c_int32(0), C.c_int32(0), C.c_int32(0)
        _lib.check(self._libh.fhtgs_context_get_blend_split_stats(self.ctx, C.byref(t), C.byref(g), C.byref(f),
                                                                   C.byref(m)))
        return dict(split_tiles=int(t.value), segments=int(g.value), whole_fallbacks=int(f.value),
                    max_records=int(m.value))

    def autotune(self, positions, scales, rotations, opacities, sh_0, sh_rest, settings: list[RasterizerSettings],
                 to_chw: bool = True, blur_periphery: bool = False, aaa_mode: bool = False, fast_math: bool = True,
                 repeats: int = 5, view_foveation: list | None = None) -> dict:
        """Times the tuning candidates on this frame and keeps the fastest (see fhtgs_autotune)."""
        keep, prims, views, st, images, n = self._frame(positions, scales, rotations, opacities, sh_0, sh_rest,
                                                        settings, to_chw, blur_periphery, aaa_mode, fast_math, None,
                                                        view_foveation)
        best = _lib.Tuning()
        ms = C.c_float(0.0)
        with torch.cuda.device(self.device):
            _lib.check(self._libh.fhtgs_autotune(self.ctx, C.byref(prims), views, len(settings), C.byref(st),
                                                 int(repeats), C.byref(best), C.byref(ms),
                                                 _stream_handle(self.device)))
        self._last_views, self._last_n = len(settings), n
        self._last_sizes = [(int(s.width), int(s.height)) for s in settings]
        return dict(blend_warp_width=int(best.blend_warp_width), blend_blocks_per_sm=int(best.blend_blocks_per_sm),
                    sort_items=int(best.sort_items), frame_ms=float(ms.value))

    def capture(self, positions, scales, rotations, opacities, sh_0, sh_rest, settings: list[RasterizerSettings],
                to_chw: bool = True, blur_periphery: bool = False, aaa_mode: bool = False, fast_math: bool = True,
                images: list[torch.Tensor] | None = None, gaze: torch.Tensor | None = None,
                capacity_headroom: float = 1.25, view_foveation: list | None = None) -> "FrameGraph":
        """Captures one frame of len(settings) views into a CUDA graph (see fhtgs_frame_graph_create).

        All tensors are used in place by every launch: update camera matrices, masks and
        Gaussians with copy_() between launches.  `gaze`: optional float32 [n_views, 2] CUDA
        tensor read at every launch (else the settings' host gaze is baked in).
        """
        keep, prims, views, st, images, n = self._frame(positions, scales, rotations, opacities, sh_0, sh_rest,
                                                        settings, to_chw, blur_periphery, aaa_mode, fast_math, images,
                                                        view_foveation)
        gptr = None
        if gaze is not None:
            if gaze.device != self.device or gaze.dtype != torch.float32 or gaze.numel() != 2 * len(settings):
                raise ValueError("gaze must be a float32 [n_views, 2] tensor on the renderer's device")
            gaze = gaze.contiguous()
            gptr = gaze.data_ptr()
            keep.refs.append(gaze)
        out = _lib.vp()
        with torch.cuda.device(self.device):
            _lib.check(self._libh.fhtgs_frame_graph_create(self.ctx, C.byref(prims), views, len(settings),
                                                           C.byref(st), gptr, float(capacity_headroom),
                                                           C.byref(out), _stream_handle(self.device)))
        self._last_views, self._last_n = len(settings), n
        self._last_sizes = [(int(s.width), int(s.height)) for s in settings]
        return FrameGraph(self, out.value, keep, images)

    def frame_info(self, view: int = 0) -> dict:
        fi = _lib.FrameInfo()
        _lib.check(self._libh.fhtgs_get_frame_info(self.ctx, view, C.byref(fi)))
        return dict(n_instances=int(fi.n_instances), instance_capacity=int(fi.instance_capacity),
                    n_active_tiles=int(fi.n_active_tiles), partition_ranges=list(fi.partition_ranges),
                    overflow=bool(fi.overflow), end_bit=int(fi.end_bit),
                    n_instances_stored=int(fi.n_instances_stored))

    def intermediates(self, view: int = 0) -> dict:
        """Host copies of the last frame's per-primitive, tile and instance data of one view."""
        import numpy as np

        info = self.frame_info(view)
        n = self._last_n
        w, h = self._last_sizes[view]
        T = 4 * ((w + 15) // 16) * ((h + 15) // 16)
        m = info["n_instances"]
        na = info["n_active_tiles"]
        out = dict(n_touched=np.zeros(n, np.uint32), screen_bounds=np.zeros((n, 4), np.uint16),
                   vpmt=np.zeros((n, 12), np.float32), rgba=np.zeros((n, 4), np.float32),
                   tile_index_map_partitioned=np.zeros(max(na, 1), np.uint32),
                   tile_type_partitioned=np.zeros(max(na, 1), np.uint8), keys=np.zeros(max(m, 1), np.uint32),
                   values=np.zeros(max(m, 1), np.uint32), instance_ranges=np.zeros((T, 2), np.uint32))

        def p(a, t):
            return a.ctypes.data_as(t)

        im = _lib.Intermediates(p(out["n_touched"], _lib.u32p), p(out["screen_bounds"], _lib.u16p),
                                p(out["vpmt"], _lib.fp), p(out["rgba"], _lib.fp),
                                p(out["tile_index_map_partitioned"], _lib.u32p),
                                p(out["tile_type_partitioned"], _lib.u8p), p(out["keys"], _lib.u32p),
                                p(out["values"], _lib.u32p), p(out["instance_ranges"], _lib.u32p))
        _lib.check(self._libh.fhtgs_copy_intermediates(self.ctx, view, C.byref(im)))
        out["tile_index_map_partitioned"] = out["tile_index_map_partitioned"][:na]
        out["tile_type_partitioned"] = out["tile_type_partitioned"][:na]
        out["keys"] = out["keys"][:m]
        out["values"] = out["values"][:m]
        out.update(info)
        return out


class FrameGraph:
    """A captured frame (fhtgs_frame_graph): `launch()` replays it on the current stream."""

    def __init__(self, renderer: Renderer, handle: int, keep, images: list[torch.Tensor]):
        self.renderer = renderer
        self.handle = handle
        self._keep = keep  # every tensor the graph reads or writes stays alive with it
        self.images = images

    def launch(self, sync: bool = False) -> list[torch.Tensor]:
        r = self.renderer
        with torch.cuda.device(r.device):
            _lib.check(r._libh.fhtgs_frame_graph_launch(self.handle, _stream_handle(r.device)))
            if sync:
                torch.cuda.current_stream(r.device).synchronize()
        return self.images

    def close(self):
        if getattr(self, "handle", None):
            self.renderer._libh.fhtgs_frame_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
