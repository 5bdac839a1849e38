"""Device-side helpers on either side of the rendering path, over the C ABI of libfhtgs.so.

* `build_tile_masks` — the three mask tensors a view needs (visibility bitmask, its
  summed-area table, the fovea table), built on the GPU from one byte per 16x16 tile.  The
  reference takes them precomputed by the calling framework
  (`torch_bindings/rasterization.py:22-43`); this builds them without a host round trip.
* `pack_display` — float images to one RGBA8/BGRA8 image, views side by side (stereo:
  left | right), for a display or encoder that wants 8-bit pixels.
* `_C_visualization` / `FoveatedHTGSVisualizer` — drop-ins for the reference's debug overlays
  (`torch_bindings/bindings_visualization.cpp:8-9`, `torch_bindings/rasterization.py:157-191`):
  `visualize_gaze` draws the gaze marker, `visualize_tile_boundaries` outlines the fovea,
  blended and periphery tiles.  Both draw into the image in place and return it.

Everything runs asynchronously on PyTorch's current stream.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib

TILE_LARGE = 16
FOVEA_TABLE_ENTRIES = 49 * 49


def _stream(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _cuda_device(device) -> torch.device:
    d = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if d.type != "cuda":
        raise ValueError(f"device must be a CUDA device, got {d}")
    if d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    return d


def grid_large(width: int, height: int) -> tuple[int, int]:
    return -(-int(width) // TILE_LARGE), -(-int(height) // TILE_LARGE)


def build_tile_masks(width: int, height: int, visible_tiles: torch.Tensor | None = None, device=None,
                     with_fovea_table: bool = True):
    """(visibility_mask, visibility_mask_area_table, fovea_mask_area_table) as torch.uint32.

    `visible_tiles`: [grid_h, grid_w] (or flat) bool/uint8 tensor on the GPU, non-zero = visible;
    None = every tile visible.  Shapes of the results: [ceil(tiles/32)], [(grid_w+1)*(grid_h+1)],
    [49*49] (None when `with_fovea_table` is false).
    """
    lib = _lib.load()
    gw, gh = grid_large(width, height)
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    dev = _cuda_device(visible_tiles.device if visible_tiles is not None else device)
    vis_ptr = None
    if visible_tiles is not None:
        if visible_tiles.numel() != gw * gh:
            raise ValueError(f"visible_tiles must hold {gh}x{gw} entries, got {tuple(visible_tiles.shape)}")
        if visible_tiles.dtype == torch.bool:
            visible_tiles = visible_tiles.view(torch.uint8)
        if visible_tiles.dtype != torch.uint8:
            raise TypeError(f"visible_tiles must be bool or uint8, got {visible_tiles.dtype}")
        visible_tiles = visible_tiles.contiguous()
        vis_ptr = visible_tiles.data_ptr()
    words = torch.empty(-(-(gw * gh) // 32), dtype=torch.uint32, device=dev)
    sat = torch.empty((gw + 1) * (gh + 1), dtype=torch.uint32, device=dev)
    fovea = torch.empty(FOVEA_TABLE_ENTRIES, dtype=torch.uint32, device=dev) if with_fovea_table else None
    _lib.check(lib.fhtgs_build_tile_masks(vis_ptr, int(width), int(height), words.data_ptr(), sat.data_ptr(),
                                          fovea.data_ptr() if fovea is not None else None, _stream(dev)))
    return words, sat, fovea


def pack_display(images, to_chw: bool = True, bgra: bool = False, out: torch.Tensor | None = None) -> torch.Tensor:
    """Packs 1..8 float32 RGB images (same size) into one [H, n*W, 4] uint8 image, side by side.

    Channels are clamped to [0, 1] (NaN -> 0) and rounded half up to 8 bits; alpha is 255.
    `bgra` swaps red and blue for displays that scan out BGRA.
    """
    lib = _lib.load()
    if isinstance(images, torch.Tensor):
        images = [images]
    images = list(images)
    if not 1 <= len(images) <= 8:
        raise ValueError("pack_display takes 1 to 8 images")
    shape = images[0].shape
    dev = _cuda_device(images[0].device)
    for im in images:
        if im.shape != shape or im.dtype != torch.float32 or im.device != dev:
            raise ValueError("images must be float32 tensors of one shape on one CUDA device")
        if not im.is_contiguous():
            raise ValueError("images must be contiguous")
    if len(shape) != 3 or shape[0 if to_chw else 2] != 3:
        raise ValueError(f"images must be {'[3,H,W]' if to_chw else '[H,W,3]'}, got {tuple(shape)}")
    h, w = (shape[1], shape[2]) if to_chw else (shape[0], shape[1])
    n = len(images)
    if out is None:
        out = torch.empty((h, n * w, 4), dtype=torch.uint8, device=dev)
    elif out.shape != (h, n * w, 4) or out.dtype != torch.uint8 or out.device != dev or not out.is_contiguous():
        raise ValueError(f"out must be a contiguous uint8 tensor of shape {(h, n * w, 4)} on {dev}")
    ptrs = (C.c_void_p * n)(*[im.data_ptr() for im in images])
    _lib.check(lib.fhtgs_pack_display(ptrs, n, int(w), int(h), int(bool(to_chw)), int(bool(bgra)), out.data_ptr(),
                                      _stream(dev)))
    return out


def _image_size(image: torch.Tensor, to_chw: bool) -> tuple[int, int]:
    if not isinstance(image, torch.Tensor) or image.dtype != torch.float32 or image.device.type != "cuda":
        raise TypeError("image must be a float32 CUDA tensor")
    if image.dim() != 3 or image.shape[0 if to_chw else 2] != 3:
        raise ValueError(f"image must be {'[3,H,W]' if to_chw else '[H,W,3]'}, got {tuple(image.shape)}")
    if not image.is_contiguous():
        raise ValueError("image must be contiguous (it is drawn into in place)")
    return int(image.shape[2 if to_chw else 1]), int(image.shape[1 if to_chw else 0])


def _host_floats(t, n: int, name: str) -> list[float]:
    t = torch.as_tensor(t).detach().reshape(-1)
    if t.numel() < n:
        raise ValueError(f"{name} needs {n} values")
    return [float(x) for x in t[:n].to("cpu", torch.float32)]


class _CVisualizationModule:
    """Positional drop-in for the reference's `_C_visualization` extension module."""

    @staticmethod
    def visualize_gaze(image: torch.Tensor, gaze_position, gaze_color, visualization_type, visualization_size: int,
                       to_chw: bool) -> torch.Tensor:
        lib = _lib.load()
        w, h = _image_size(image, to_chw)
        gx, gy = _host_floats(gaze_position, 2, "gaze_position")
        r, g, b = _host_floats(gaze_color, 3, "gaze_color")
        vt = int(getattr(visualization_type, "value", visualization_type))
        _lib.check(lib.fhtgs_visualize_gaze(image.data_ptr(), w, h, gx, gy, r, g, b, vt, int(visualization_size),
                                            int(bool(to_chw)), _stream(image.device)))
        return image

    @staticmethod
    def visualize_tile_boundaries(image: torch.Tensor, visibility_mask: torch.Tensor, gaze_position,
                                  to_chw: bool) -> torch.Tensor:
        lib = _lib.load()
        w, h = _image_size(image, to_chw)
        gw, gh = grid_large(w, h)
        if not isinstance(visibility_mask, torch.Tensor) or visibility_mask.device != image.device:
            raise ValueError("visibility_mask must be a tensor on the image's device")
        if visibility_mask.dtype not in (torch.uint32, torch.int32):
            raise TypeError(f"visibility_mask must be uint32 (or int32 bit pattern), got {visibility_mask.dtype}")
        if visibility_mask.numel() < -(-(gw * gh) // 32):
            raise ValueError(f"visibility_mask needs {-(-(gw * gh) // 32)} words for a {w}x{h} image")
        mask = visibility_mask.contiguous()
        gx, gy = _host_floats(gaze_position, 2, "gaze_position")
        _lib.check(lib.fhtgs_visualize_tile_boundaries(image.data_ptr(), w, h, mask.data_ptr(), gx, gy,
                                                       int(bool(to_chw)), _stream(image.device)))
        return image


_C_visualization = _CVisualizationModule()


class FoveatedHTGSVisualizer(torch.nn.Module):
    """Mirror of the reference's `FoveatedHTGSVisualizer` (`torch_bindings/rasterization.py:157-191`)."""

    def visualize_gaze(self, image, gaze_position, gaze_color, visualization_size: int, visualization_type,
                       to_chw: bool) -> torch.Tensor:
        return _C_visualization.visualize_gaze(image, gaze_position, gaze_color, visualization_type,
                                               visualization_size, to_chw)

    def visualize_tile_boundaries(self, image, visibility_mask, gaze_position, to_chw: bool) -> torch.Tensor:
        return _C_visualization.visualize_tile_boundaries(image, visibility_mask, gaze_position, to_chw)
