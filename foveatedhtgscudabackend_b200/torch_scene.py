"""Conversion of the NumPy scenes/views of `scene.py` into the tensors the API consumes."""
from __future__ import annotations

import numpy as np
import torch

from . import scene as _scene
from .rasterization import BackgroundModel, RasterizerSettings


def gaussians_to_torch(g: _scene.Gaussians, device="cuda", storage: str = "fp32") -> tuple[torch.Tensor, ...]:
    """(positions, scales, rotations, opacities, sh_0, sh_rest) on `device`.

    storage "fp32": every attribute float32.  "half": positions float32; scales, rotations and
    opacities float16; sh_0 and sh_rest bfloat16 (rounded to nearest even from float32).
    """
    def t(a):
        return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)
    out = (t(g.positions), t(g.scales), t(g.rotations), t(g.opacities), t(g.sh_0), t(g.sh_rest))
    if storage == "fp32":
        return out
    if storage != "half":
        raise ValueError(f"unknown storage {storage!r}")
    return to_half_storage(*out)


def to_half_storage(positions, scales, rotations, opacities, sh_0, sh_rest) -> tuple[torch.Tensor, ...]:
    """The reduced-precision storage of float32 Gaussians (see gaussians_to_torch)."""
    return (positions.float().contiguous(), scales.half().contiguous(), rotations.half().contiguous(),
            opacities.half().contiguous(), sh_0.bfloat16().contiguous(), sh_rest.bfloat16().contiguous())


def from_half_storage(positions, scales, rotations, opacities, sh_0, sh_rest) -> tuple[torch.Tensor, ...]:
    """Float32 copies of reduced-precision Gaussians (exact widening)."""
    return tuple(x.float().contiguous() for x in (positions, scales, rotations, opacities, sh_0, sh_rest))


def settings_from_view(v: _scene.View, *, K: int = 8, active_sh_bases: int = 16, scale_modifier: float = 1.0,
                       background: BackgroundModel = BackgroundModel.NONE, background_data=None,
                       device="cuda") -> RasterizerSettings:
    """RasterizerSettings for a scene.View; gaze stays on the host like the reference wants."""
    def f(a):
        return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)

    def u(a):  # torch.uint32: the reference's bindings read these with data_ptr<uint>()
        return torch.from_numpy(np.ascontiguousarray(a, np.uint32)).to(device)

    bg = np.zeros((1,), np.float32) if background_data is None else background_data
    return RasterizerSettings(
        M=f(v.M), VPM=f(v.VPM), VPR_inv=f(v.VPR_inv), cam_position=f(v.cam_position),
        gaze_position=torch.from_numpy(np.ascontiguousarray(v.gaze_position, np.float32)),
        visibility_mask=u(v.visibility_mask), visibility_mask_area_table=u(v.visibility_mask_area_table),
        fovea_mask_area_table=u(v.fovea_mask_area_table), background_model_data=f(bg),
        background_model=background, K=K, active_sh_bases=active_sh_bases, width=v.width, height=v.height,
        focal_x=v.focal_x, focal_y=v.focal_y, center_x=v.center_x, center_y=v.center_y,
        near_plane=v.near_plane, far_plane=v.far_plane, scale_modifier=scale_modifier)
