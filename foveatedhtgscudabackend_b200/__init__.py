"""B200-native forward renderer for foveated hybrid-transparency Gaussian splatting.

Drop-in for the rasterization path of TrueKuehli/FoveatedHTGSCudaBackend: the same
`FoveatedHTGSRasterizer` / `RasterizerSettings` surface and the same positional `_C`,
`_C_benchmarking`, `_C_stereo` and `_C_visualization` entry points, backed by libfhtgs.so (hand-written sm_100a
kernels behind the C ABI in include/fhtgs.h).
"""
from .rasterization import (  # noqa: F401
    BackgroundModel,
    FoveatedHTGSRasterizer,
    GazeVisualizationType,
    RasterizerSettings,
    FrameGraph,
    Renderer,
    _C,
    _C_benchmarking,
    _C_stereo,
)
from ._lib import FhtgsError  # noqa: F401
from .serving import Completion, Server, ServerGroup  # noqa: F401
from .display import FoveatedHTGSVisualizer, _C_visualization, build_tile_masks, pack_display  # noqa: F401
from .torch_scene import from_half_storage, gaussians_to_torch, settings_from_view, to_half_storage  # noqa: F401

__all__ = ["FoveatedHTGSRasterizer", "FoveatedHTGSVisualizer", "RasterizerSettings", "BackgroundModel",
           "GazeVisualizationType", "Renderer", "FhtgsError", "gaussians_to_torch", "settings_from_view",
           "build_tile_masks", "pack_display", "Server", "ServerGroup", "Completion"]
