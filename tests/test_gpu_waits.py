"""The bounded device-side waits of a frame run out without a fault, are reported with the stage
that gave up, and leave the context usable.

Two stages wait on the device: the instance sort's decoupled look-back (a tile reads the digit
counts that earlier tiles publish) and the preprocess's wait for the bulk copies that stage a
block's Gaussians in shared memory.  fhtgs_context_test_wait_timeout arms one frame so that one
of them runs out: the sort's first pass never hands out tile 0 (its counts are never published,
a flag nothing sets), or the staging wait gives up before its copies can land.  Each test checks
that the frame returns within its limit with FHTGS_ERR_CUDA naming the stage, that the failed
view renders background only (its range stage skipped the unpublished order), and that the next
frame on the same context is bit-identical to one rendered before the test.  Nothing faults,
traps or hangs the GPU: every wait is bounded and the kernels return after recording the error.
"""
import ctypes as C
import time

import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import _lib, scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def frame():
    # 40k SH3 Gaussians, two 640x480 eyes: well over one sort tile (4096 pairs) per eye, and
    # full preprocess blocks of 16-byte aligned fp32 arrays (the staged fast-math path)
    g = scene.make_gaussians(40_000, 3, seed=5)
    views = scene.make_stereo_views(640, 480, seed=1)
    gt = F.gaussians_to_torch(g, "cuda:0")
    st = [F.settings_from_view(v, K=8, active_sh_bases=16, device="cuda:0") for v in views]
    return gt, st, views


def render(r, frame, sync=True):
    gt, st, views = frame
    imgs = [torch.zeros((3, v.height, v.width), device="cuda:0") for v in views]
    r.render(*gt, st, to_chw=True, fast_math=True, images=imgs, sync=sync)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in imgs]


def arm(r, which, limit):
    _lib.check(r._libh.fhtgs_context_test_wait_timeout(r.ctx, which, limit))


# The staging wait is tested with a limit of 0 polls (it gives up before it looks): a single
# mbarrier poll may suspend the thread until the copies land, so any larger limit may not run out.
@pytest.mark.parametrize("which,limit,stage", [
    (_lib.WAIT_TEST_SORT_LOOKBACK, 10_000, "look-back"),
    (_lib.WAIT_TEST_STAGING, 0, "staging"),
])
def test_wait_runs_out_is_reported_and_the_next_frame_is_exact(frame, which, limit, stage):
    r = F.Renderer("cuda:0")
    try:
        before = render(r, frame)
        n_stored = [r.frame_info(i)["n_instances_stored"] for i in range(2)]
        assert min(n_stored) > 4096  # tile 1 of the first sort pass exists

        arm(r, which, limit)
        t0 = time.perf_counter()
        with pytest.raises(_lib.FhtgsError) as err:
            render(r, frame, sync=True)
        elapsed = time.perf_counter() - t0
        assert err.value.status == 2 and stage in str(err.value)
        assert elapsed < 10.0, f"the frame took {elapsed:.1f} s to give up"
        # the asynchronous path reports the same through fhtgs_get_frame_info
        arm(r, which, limit)
        failed = render(r, frame, sync=False)
        fi = _lib.FrameInfo()
        st = r._libh.fhtgs_get_frame_info(r.ctx, 0, C.byref(fi))
        assert st == 2 and stage in r._libh.fhtgs_last_error().decode()
        # a failed view is background only (the default background is black): nothing blended
        assert all(float(np.abs(img).max()) == 0.0 for img in failed)

        after = render(r, frame)
        for a, b in zip(before, after):
            assert np.array_equal(a, b)
        assert [r.frame_info(i)["n_instances_stored"] for i in range(2)] == n_stored
    finally:
        r.close()


def test_wait_test_arguments_are_checked():
    r = F.Renderer("cuda:0")
    try:
        lib = r._libh
        assert lib.fhtgs_context_test_wait_timeout(r.ctx, 3, 0) == 1
        assert lib.fhtgs_context_test_wait_timeout(r.ctx, _lib.WAIT_TEST_STAGING, -1) == 1
        assert lib.fhtgs_context_test_wait_timeout(r.ctx, _lib.WAIT_TEST_SORT_LOOKBACK, 1 << 23) == 1
        assert lib.fhtgs_context_test_wait_timeout(None, _lib.WAIT_TEST_STAGING, 0) == 1
    finally:
        r.close()
