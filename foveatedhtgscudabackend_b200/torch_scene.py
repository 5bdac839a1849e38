"""Conversion of the NumPy scenes/views of `scene.py` into the tensors the API consumes."""
from __future__ import annotations

import numpy as np
import torch

from . import scene as _scene
from .rasterization import BackgroundModel, RasterizerSettings


def gaussians_to_torch(g: _scene.Gaussians, device="cuda") -> tuple[torch.Tensor, ...]:
    """(positions, scales, rotations, opacities, sh_0, sh_rest) as float32 tensors on `device`."""
    def t(a):
        return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)
    return (t(g.positions), t(g.scales), t(g.rotations), t(g.opacities), t(g.sh_0), t(g.sh_rest))


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
