"""GPU tests of batched frames through the C ABI: many mixed-resolution views in one frame, the
tuning variants, the autotuner and captured frame graphs.

Every check is bit-exact: a view rendered inside a batch, with any tuning, or by replaying a
captured graph must equal the same view rendered alone by the default eager path.
"""
import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import _lib, scene

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
RES = ((160, 120), (320, 200), (272, 400), (96, 64))


@pytest.fixture(scope="module")
def batch():
    g = scene.make_gaussians(40000, 3, seed=21)
    views = scene.make_batched_views(8, seed=3, radius=(3.0, 6.0), resolutions=RES)
    gt = F.gaussians_to_torch(g)
    st = [F.settings_from_view(v, K=8, active_sh_bases=16) for v in views]
    return gt, st


def render_alone(gt, st, **kw):
    r = F.Renderer(DEV)
    try:
        return [r.render(*gt, [s], **kw)[0].clone() for s in st]
    finally:
        r.close()


def test_batch_equals_views_rendered_alone(batch):
    gt, st = batch
    alone = render_alone(gt, st)
    r = F.Renderer(DEV)
    together = r.render(*gt, st)
    for i, (a, b) in enumerate(zip(alone, together)):
        assert torch.equal(a, b), f"view {i} differs inside the batch"
    r.close()


@pytest.mark.parametrize("width", [8, 16, 4])
@pytest.mark.parametrize("blocks", [0, 2])
@pytest.mark.parametrize("items", [16, 12, 8])
def test_every_tuning_renders_identical_images(batch, width, blocks, items):
    gt, st = batch
    ref = F.Renderer(DEV)
    expect = [x.clone() for x in ref.render(*gt, st)]
    ref.close()
    r = F.Renderer(DEV)
    r.set_tuning(width, blocks, items)
    assert r.get_tuning() == dict(blend_warp_width=width, blend_blocks_per_sm=blocks, sort_items=items)
    got = r.render(*gt, st)
    for i, (a, b) in enumerate(zip(expect, got)):
        assert torch.equal(a, b), f"view {i} differs with tuning {width}/{blocks}/{items}"
    # the sorted instances are the same too
    for v in range(len(st)):
        assert r.frame_info(v)["n_instances_stored"] == ref_info(gt, st, v)
    r.close()


_ref_counts = {}


def ref_info(gt, st, v):
    key = v
    if key not in _ref_counts:
        r = F.Renderer(DEV)
        r.render(*gt, st)
        for i in range(len(st)):
            _ref_counts[i] = r.frame_info(i)["n_instances_stored"]
        r.close()
    return _ref_counts[key]


def test_bad_tuning_is_rejected():
    r = F.Renderer(DEV)
    for bad in ((5, 0, 16), (8, 9, 16), (8, 0, 10)):
        with pytest.raises(F.FhtgsError):
            r.set_tuning(*bad)
    r.close()


def test_autotune_picks_a_valid_tuning_and_keeps_images(batch):
    gt, st = batch
    expect = render_alone(gt, st)
    r = F.Renderer(DEV)
    best = r.autotune(*gt, st, repeats=2)
    assert best["blend_warp_width"] in (4, 8, 16) and best["sort_items"] in (8, 12, 16)
    assert best["blend_blocks_per_sm"] in (0, 2, 3) and best["frame_ms"] > 0
    assert {k: best[k] for k in ("blend_warp_width", "blend_blocks_per_sm", "sort_items")} == r.get_tuning()
    got = r.render(*gt, st)
    for a, b in zip(expect, got):
        assert torch.equal(a, b)
    r.close()


def test_graph_replay_equals_eager_and_follows_in_place_updates(batch):
    gt, st = batch
    r = F.Renderer(DEV)
    n = len(st)
    # device-side gaze, camera matrices updated in place between launches
    gaze = torch.stack([s.gaze_position for s in st]).to(DEV)
    live = [s._replace(M=s.M.clone(), VPM=s.VPM.clone(), VPR_inv=s.VPR_inv.clone(),
                       cam_position=s.cam_position.clone()) for s in st]
    graph = r.capture(*gt, live, gaze=gaze, capacity_headroom=2.0)
    launches_before = r.launch_count()
    imgs = graph.launch(sync=True)
    assert r.launch_count() > launches_before
    for a, b in zip(render_alone(gt, st), imgs):
        assert torch.equal(a, b)
    # move every camera (another seed's poses at the same resolutions) and every gaze
    other = scene.make_batched_views(n, seed=4, radius=(3.0, 6.0), resolutions=RES)
    rng = np.random.default_rng(5)
    moved = [F.settings_from_view(scene.make_view(int(s.width), int(s.height), position=tuple(o.cam_position),
                                                  gaze_ndc=tuple(rng.uniform(-0.8, 0.8, 2))), K=8, active_sh_bases=16)
             for s, o in zip(live, other)]
    for s, m in zip(live, moved):
        s.M.copy_(m.M)
        s.VPM.copy_(m.VPM)
        s.VPR_inv.copy_(m.VPR_inv)
        s.cam_position.copy_(m.cam_position)
    new_gaze = torch.stack([m.gaze_position for m in moved]).to(DEV)
    gaze.copy_(new_gaze)
    imgs = graph.launch(sync=True)
    for i in range(n):
        assert not r.frame_info(i)["overflow"]
    expect = render_alone(gt, [s._replace(gaze_position=m.gaze_position) for s, m in zip(live, moved)])
    for i, (a, b) in enumerate(zip(expect, imgs)):
        assert torch.equal(a, b), f"view {i} differs after the in-place update"
    graph.close()
    r.close()


def test_graph_overflow_is_flagged_not_written():
    # 300k Gaussians: about 1-2 tiles each seen from 20 units away (capacity stays at its
    # 2^20 floor), dozens of tiles each from 1.5 units: several million instances
    gt = F.gaussians_to_torch(scene.make_gaussians(300000, 0, seed=8))
    r = F.Renderer(DEV)
    far = F.settings_from_view(scene.make_view(2064, 2208, position=(0.0, 0.0, -20.0)), K=8, active_sh_bases=1)
    live = far._replace(M=far.M.clone(), VPM=far.VPM.clone(), VPR_inv=far.VPR_inv.clone(),
                        cam_position=far.cam_position.clone())
    graph = r.capture(*gt, [live], capacity_headroom=1.0)
    assert not r.frame_info(0)["overflow"]
    near = F.settings_from_view(scene.make_view(2064, 2208, position=(0.0, 0.0, -1.5)), K=8, active_sh_bases=1)
    for k in ("M", "VPM", "VPR_inv", "cam_position"):
        getattr(live, k).copy_(getattr(near, k))
    graph.launch(sync=True)
    info = r.frame_info(0)
    assert info["overflow"] and info["n_instances_stored"] > info["instance_capacity"]
    graph.close()
    r.close()


def test_graph_refuses_to_run_after_the_arena_moved(batch):
    gt, st = batch
    r = F.Renderer(DEV)
    graph = r.capture(*gt, st[:2])
    graph.launch(sync=True)
    big = [F.settings_from_view(scene.make_view(2064, 2208), K=8, active_sh_bases=16)] * 3
    r.render(*gt, big)  # a larger frame grows (moves) the arena
    with pytest.raises(F.FhtgsError) as e:
        graph.launch()
    assert e.value.status == 5
    graph.close()
    r.close()


def test_frames_in_flight_on_two_contexts_equal_one_at_a_time(batch):
    """Two contexts on two streams with frames issued round robin (frames in flight, as the
    benchmark runs them) render every frame exactly as one context does one frame at a time."""
    gt, st = batch
    alone = [x.cpu() for x in render_alone(gt, st[:2])]
    rs = [F.Renderer(DEV), F.Renderer(DEV)]
    streams = [torch.cuda.Stream(DEV), torch.cuda.Stream(DEV)]
    out = [[torch.empty_like(x, device=DEV) for x in alone] for _ in range(2)]
    try:
        for k in range(6):
            i = k % 2
            with torch.cuda.stream(streams[i]):
                rs[i].render(*gt, st[:2], images=out[i], sync=False)
        torch.cuda.synchronize()
        for i in range(2):
            for a, b in zip(alone, out[i]):
                assert torch.equal(a, b.cpu())
    finally:
        for r in rs:
            r.close()
