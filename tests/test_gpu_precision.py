"""GPU tests of reduced-precision Gaussian storage (fp16 scales/rotations/opacities, bf16 SH,
fp32 positions and arithmetic) through the C ABI.

Exactness: the half-storage path widens every attribute to float32 on load and then runs the
float32 arithmetic, so its images must equal, bit for bit, the float32 path's images of the
widened scene.  Accuracy: against the float32 scene (the storage's quantisation error) and
against the CPU FP64 oracle; the measured figures are printed and bounded here.
"""
import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
import oracle as O
from foveatedhtgscudabackend_b200 import scene
from helpers import max_abs, psnr

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.mark.parametrize("fast_math,aaa", [(True, False), (False, False), (True, True)])
def test_half_storage_equals_fp32_path_on_widened_scene(fast_math, aaa):
    g = scene.make_gaussians(60000, 3, seed=31)
    left, right = scene.make_stereo_views(640, 480, seed=2)
    st = [F.settings_from_view(v, K=8, active_sh_bases=16) for v in (left, right)]
    half = F.gaussians_to_torch(g, DEV, storage="half")
    assert half[1].dtype == torch.float16 and half[4].dtype == torch.bfloat16 and half[0].dtype == torch.float32
    widened = F.from_half_storage(*half)
    r = F.Renderer(DEV)
    a = [x.clone() for x in r.render(*half, st, fast_math=fast_math, aaa_mode=aaa)]
    b = r.render(*widened, st, fast_math=fast_math, aaa_mode=aaa)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    r.close()


def test_half_storage_accuracy_vs_fp32_and_fp64_oracle():
    g = scene.make_gaussians(40000, 3, seed=32)
    v = scene.make_view(480, 400, gaze_ndc=(0.1, -0.1))
    s = F.settings_from_view(v, K=8, active_sh_bases=16)
    r = F.Renderer(DEV)
    full = r.render(*F.gaussians_to_torch(g, DEV), [s], fast_math=False)[0].cpu().numpy()
    half = r.render(*F.gaussians_to_torch(g, DEV, storage="half"), [s], fast_math=False)[0].cpu().numpy()
    r.close()
    ref64 = O.render(g, v, K=8, active_sh_bases=16, precision=64)
    res = {"half_vs_fp32": (psnr(half, full), max_abs(half, full)),
           "fp32_vs_fp64": (psnr(full, ref64), max_abs(full, ref64)),
           "half_vs_fp64": (psnr(half, ref64), max_abs(half, ref64))}
    print("precision PSNR dB / max-abs:", {k: (round(p, 2), round(m, 5)) for k, (p, m) in res.items()})
    assert res["fp32_vs_fp64"][0] >= 50.0
    assert res["half_vs_fp32"][0] >= 35.0
    assert res["half_vs_fp64"][0] >= 35.0


def test_mixed_dtypes_are_rejected():
    g = scene.make_gaussians(100, 1, seed=1)
    v = scene.make_view(64, 64)
    s = F.settings_from_view(v, K=4, active_sh_bases=4)
    half = list(F.gaussians_to_torch(g, DEV, storage="half"))
    half[4] = half[4].float()  # sh_0 must be bf16 in the half format
    r = F.Renderer(DEV)
    with pytest.raises(TypeError):
        r.render(*half, [s])
    r.close()
