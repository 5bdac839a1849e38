"""Adversarial parity cases against the live reference (oracle/_ref): the inputs where the
blend's warp culling, the alpha thresholds and the preprocess's culling are closest to their
edges.

The blend skips a (warp rectangle, Gaussian) pair when the Gaussian's cutoff conic, with its
radius inflated by 0.5 % and the rectangle by 0.02 px, misses the rectangle: a pair it skips can
only hold fragments with alpha < 1/255, which the reference's blend drops anyway.  These scenes
put many fragments right at that edge:
  faint       opacities in [1/255, 1.05/255]: the cutoff ellipse shrinks to a point, alpha hovers
              around the 1/255 test;
  needles     scale ratios of 1.2e3 (needles) and sub-pixel splats (1e-4), bright: thin ellipses
              that cross warp rectangles between pixel centres;
  near_plane  Gaussians whose centres lie around the near plane (view z 0.1-0.3 for near 0.2):
              culled or not by the preprocess, projected with large, ill-conditioned planes;
  inside      the camera inside large Gaussians: the cutoff box is unbounded and culling is off.
Each kind at K = 1, 8, 32, with the IEEE arithmetic of `_C` and the fast-math arithmetic of
`_C_benchmarking`, gaze at the image corners.  Integer intermediates (touched counts, bounds,
tile maps, sorted keys and values, ranges) must be bit-identical; so must the image, whenever
the reference reproduces its own image (the reference skips its sort for some instance counts,
then the oracle judges: >= 80 dB).  The count of differing pixels is part of the failure
message.
"""
import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import scene
import oracle as O
import ref as REF
from helpers import assert_instances_equal, assert_tiles_equal, max_abs, psnr
from test_gpu_parity import assert_primitives_equal

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not REF.available(), reason="reference build (oracle/_ref) not present")]

W, H = 640, 480


def adversarial(kind: str, seed: int) -> scene.Gaussians:
    g = scene.make_gaussians(24000, 3, seed=seed)
    rng = np.random.default_rng(seed + 1000)
    n = g.n
    if kind == "faint":
        sel = rng.random(n) < 0.6
        g.opacities[sel, 0] = rng.uniform(1.0 / 255.0, 1.05 / 255.0, int(sel.sum())).astype(np.float32)
        g.scales[sel] *= 6.0  # wide enough to cover several tiles
    elif kind == "needles":
        sel = rng.random(n) < 0.5
        s = g.scales[sel]
        s[:, 0] *= 30.0
        s[:, 1:] /= 40.0
        g.scales[sel] = s
        tiny = (~sel) & (rng.random(n) < 0.4)
        g.scales[tiny] = 1e-4
        g.opacities[sel | tiny, 0] = rng.uniform(0.3, 0.99, int((sel | tiny).sum())).astype(np.float32)
    elif kind == "near_plane":
        k = n // 3
        idx = rng.choice(n, k, replace=False)
        pos = np.stack([rng.uniform(-0.15, 0.15, k), rng.uniform(-0.1, 0.1, k), rng.uniform(-5.9, -5.7, k)], 1)
        g.positions[idx] = pos.astype(np.float32)
        g.scales[idx] = np.exp(rng.normal(-3.5, 0.6, (k, 3))).astype(np.float32)
    elif kind == "inside":
        k = 200
        idx = rng.choice(n, k, replace=False)
        g.positions[idx] = (np.array([0.0, 0.0, -6.0]) + rng.normal(0.0, 0.25, (k, 3))).astype(np.float32)
        g.scales[idx] = rng.uniform(0.4, 2.0, (k, 3)).astype(np.float32)
        g.opacities[idx, 0] = rng.uniform(0.01, 0.3, k).astype(np.float32)
    else:
        raise ValueError(kind)
    return g


CASES = [(kind, K, fast) for kind in ("faint", "needles", "near_plane", "inside") for K in (1, 8, 32)
         for fast in (True, False)]


@pytest.fixture(scope="module")
def renderer():
    r = F.Renderer("cuda:0")
    yield r
    r.close()


@pytest.mark.parametrize("kind,K,fast", CASES, ids=[f"{k}-K{K}-{'fast' if f else 'ieee'}" for k, K, f in CASES])
def test_adversarial_vs_live_reference(renderer, kind, K, fast):
    seed = {"faint": 301, "needles": 302, "near_plane": 303, "inside": 304}[kind]
    g = adversarial(kind, seed)
    corner = (-1.0, -1.0) if (K + int(fast)) % 2 == 0 else (1.0, 1.0)
    v = scene.make_view(W, H, gaze_ndc=corner)
    gt = F.gaussians_to_torch(g)
    st = F.settings_from_view(v, K=K, active_sh_bases=16)
    mine = renderer.render(*gt, [st], to_chw=True, fast_math=fast)[0]
    torch.cuda.synchronize()
    mine = mine.cpu().numpy()
    inter = renderer.intermediates(0)
    what = f"{kind}/K{K}/{'fast' if fast else 'ieee'}"
    ref = REF.intermediates(gt, st, fast=fast)
    assert_primitives_equal(inter, ref, what)
    assert_tiles_equal(inter, ref, what)
    assert_instances_equal(inter, ref, ref["end_bit"], what)

    mod = REF.module("_C_benchmarking" if fast else "_C")
    call = mod.benchmark if fast else mod.render

    def ref_image():
        out = call(*gt, *st.as_tuple(), True, False, False)
        torch.cuda.synchronize()
        return out.cpu().numpy()

    first, second = ref_image(), ref_image()
    if np.array_equal(first, second):
        differ = int(np.count_nonzero((mine != first).any(0)))
        print(f"adversarial {what}: {differ} pixels differ from the live reference")
        assert differ == 0, (f"{what}: {differ} of {W * H} pixels differ from the reference "
                             f"(max-abs {max_abs(mine, first):.3g}, PSNR {psnr(mine, first):.1f} dB)")
    else:
        p = psnr(mine, O.render(g, v, K=K, active_sh_bases=16, precision=32))
        print(f"adversarial {what}: reference not reproducible; {p:.1f} dB against the oracle")
        assert p >= 80.0, f"{what}: reference not reproducible; PSNR vs oracle {p:.1f} dB"
