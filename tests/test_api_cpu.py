"""Drop-in Python surface: names, field order and argument checking (no GPU)."""
import pytest
import torch

import foveatedhtgscudabackend_b200 as F


def test_rasterizer_settings_field_order_matches_reference():
    # torch_bindings/rasterization.py:22-43 of the reference
    assert F.RasterizerSettings._fields == (
        "M", "VPM", "VPR_inv", "cam_position", "gaze_position", "visibility_mask", "visibility_mask_area_table",
        "fovea_mask_area_table", "background_model_data", "background_model", "K", "active_sh_bases", "width",
        "height", "focal_x", "focal_y", "center_x", "center_y", "near_plane", "far_plane", "scale_modifier")
    assert [m.value for m in F.BackgroundModel] == [0, 1, 2, 3]


def test_as_tuple_passes_enum_value():
    s = F.RasterizerSettings(*([torch.zeros(1)] * 9), F.BackgroundModel.TEXTURE, 8, 16, 64, 48, 1.0, 1.0, 32.0, 24.0,
                             0.2, 100.0, 1.0)
    t = s.as_tuple()
    assert len(t) == 21 and t[9] == 2 and t[10] == 8


def test_positional_arity_checked():
    with pytest.raises(TypeError):
        F._C.render(*([None] * 29))
    with pytest.raises(TypeError):
        F._C_benchmarking.benchmark(*([None] * 31))
    with pytest.raises(TypeError):
        F._C_stereo.render(*([None] * 50))


def test_cpu_tensors_rejected_before_any_device_work():
    x = torch.zeros(4, 3)
    with pytest.raises(ValueError):
        F._C.render(x, *([None] * 29))


def test_rasterizer_is_module():
    r = F.FoveatedHTGSRasterizer()
    assert isinstance(r, torch.nn.Module)
    assert hasattr(r, "render") and hasattr(r, "benchmark") and hasattr(r, "render_stereo")
