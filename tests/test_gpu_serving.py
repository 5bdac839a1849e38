"""GPU tests of the request server (fhtgs_server_*): continuous batching over resident scenes,
HBM-budget admission, server-owned outputs and overflow re-renders.

Tolerance: none.  A request's images must equal, bit for bit, the images of the same views
rendered alone by `Renderer.render` and by the drop-in `_C_stereo.render`, whether the request
ran alone or fused into a frame with other requests (max-abs 2e-3 and PSNR
>= 50 dB; batching is exact, so the test asks for equality).
"""
import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import _lib, scene
from foveatedhtgscudabackend_b200.serving import Server

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
RES = ((320, 240), (480, 400), (272, 208))


@pytest.fixture(scope="module")
def scenes():
    out = []
    for n, seed, deg in ((30000, 1, 3), (60000, 2, 3), (15000, 3, 0)):
        g = scene.make_gaussians(n, deg, seed=seed)
        out.append((F.gaussians_to_torch(g, DEV), (deg + 1) ** 2))
    return out


def make_requests(n: int, n_scenes: int, seed: int = 0):
    """(scene index, [left, right]) stereo requests of mixed resolution, pose and gaze."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        w, h = RES[int(rng.integers(len(RES)))]
        d = rng.normal(size=3)
        d[1] *= 0.3
        d /= np.linalg.norm(d)
        pos = tuple(rng.uniform(4.0, 7.0) * d)
        g = tuple(rng.uniform(-0.5, 0.5, size=2))
        left = scene.make_view(w, h, position=pos, eye_offset=-0.0315, gaze_ndc=g)
        right = scene.make_view(w, h, position=pos, eye_offset=+0.0315, gaze_ndc=g)
        reqs.append((i % n_scenes, [left, right]))
    return reqs


def render_reference(scenes, reqs):
    """Each request rendered alone by the drop-in stereo call (blocking, fresh output tensors)."""
    out = []
    for si, (left, right) in reqs:
        gt, active = scenes[si]
        st = [F.settings_from_view(v, K=8, active_sh_bases=active, device=DEV) for v in (left, right)]
        a, b = F._C_stereo.render(*gt, *st[0].as_tuple(), *st[1].as_tuple(), True, False, False)
        out.append((a.clone(), b.clone()))
    return out


def serve(srv, ids, reqs, alone: bool):
    """Submits every request (all at once, or each after the previous completed); returns the
    images by request index and the completions."""
    got, comps = {}, []
    tickets = {}

    def collect(cs):
        for c in cs:
            assert c.ok, f"request {c.tag} failed: {c.message}"
            got[c.tag] = tuple(x.clone() for x in c.images)
            srv.release(c.ticket)
            comps.append(c)

    if not alone:
        srv.pause()  # the whole burst reaches the batcher at once
    for k, (si, eyes) in enumerate(reqs):
        tickets[srv.submit(ids[si], eyes, tag=k)] = k
        if alone:
            cs = []
            while not cs:
                cs = srv.poll(wait_ms=2000)
            collect(cs)
    if not alone:
        srv.resume()
    while len(got) < len(reqs):
        cs = srv.poll(wait_ms=5000)
        assert cs, "server made no progress"
        collect(cs)
    return got, comps


def add_all(srv, scenes):
    return [srv.add_scene(*gt, K=8, active_sh_bases=active) for gt, active in scenes]


def test_each_result_is_the_same_alone_and_in_the_mix(scenes):
    reqs = make_requests(14, len(scenes), seed=5)
    ref = render_reference(scenes, reqs)
    # queued requests of a scene are fused into one frame (up to 8 per frame)
    with Server(DEV, max_in_flight=2, max_batch_requests=8) as srv:
        ids = add_all(srv, scenes)
        alone, _ = serve(srv, ids, reqs, alone=True)
        mixed, comps = serve(srv, ids, reqs, alone=False)
        st = srv.stats()
    assert st["max_frame_requests"] >= 4, "queued requests of a scene were not batched"
    assert max(c.frame_views for c in comps) >= 8
    assert st["failed"] == 0 and st["completed"] == 2 * len(reqs)
    for k in range(len(reqs)):
        for e in range(2):
            assert torch.equal(alone[k][e], ref[k][e]), f"request {k} eye {e}: served alone != drop-in call"
            assert torch.equal(mixed[k][e], ref[k][e]), f"request {k} eye {e}: served in the mix != drop-in call"


def test_overlapping_slots_and_caller_images(scenes):
    """Three slots in flight, outputs in caller-owned tensors; same images as the drop-in call."""
    reqs = make_requests(12, len(scenes), seed=9)
    ref = render_reference(scenes, reqs)
    with Server(DEV, max_in_flight=3, max_batch_requests=4) as srv:
        ids = add_all(srv, scenes)
        outs = []
        for k, (si, eyes) in enumerate(reqs):
            imgs = [torch.full((3, v.height, v.width), -1.0, device=DEV) for v in eyes]
            outs.append(imgs)
            srv.submit(ids[si], eyes, images=imgs, tag=k)
        srv.drain(timeout_ms=60000)
        comps = srv.poll(max_completions=64)
        st = srv.stats()
    assert len(comps) == len(reqs) and all(c.ok for c in comps)
    assert st["queued"] == 0 and st["in_flight"] == 0
    for c in comps:
        assert c.done_ms >= c.launch_ms >= c.submit_ms
        assert c.images[0].data_ptr() == outs[c.tag][0].data_ptr()
    for k in range(len(reqs)):
        for e in range(2):
            assert torch.equal(outs[k][e], ref[k][e]), f"request {k} eye {e} differs"


def test_settings_eyes_with_partial_masks(scenes):
    """Eyes given as RasterizerSettings carry their own mask tables (here: a lens mask)."""
    gt, active = scenes[0]
    w, h = 320, 240
    gw, gh = -(-w // 16), -(-h // 16)
    vis = scene.lens_visibility(gw, gh)
    left = scene.make_view(w, h, eye_offset=-0.0315, visible=vis)
    right = scene.make_view(w, h, eye_offset=0.0315, visible=vis)
    st = [F.settings_from_view(v, K=8, active_sh_bases=active, device=DEV) for v in (left, right)]
    a, b = F._C_stereo.render(*gt, *st[0].as_tuple(), *st[1].as_tuple(), True, False, False)
    with Server(DEV) as srv:
        sid = srv.add_scene(*gt, K=8, active_sh_bases=active)
        srv.submit(sid, st)                 # settings eyes
        srv.submit(sid, [left, right])      # scene.View eyes with a partial mask
        srv.drain(timeout_ms=30000)
        comps = srv.poll()
        assert len(comps) == 2 and all(c.ok for c in comps)
        # server-owned outputs live until release() or close(): compare them before either
        for c in comps:
            assert torch.equal(c.images[0], a) and torch.equal(c.images[1], b)


def test_budget_admission(scenes):
    gt, active = scenes[1]
    reqs = make_requests(6, 1, seed=3)
    ref = render_reference([scenes[1]], reqs)
    # learn what one frame of the largest request needs, then allow a little more than that
    big = max(range(len(reqs)), key=lambda k: reqs[k][1][0].width * reqs[k][1][0].height)
    with Server(DEV, max_in_flight=2, max_batch_requests=1) as probe:
        sid = probe.add_scene(*gt, K=8, active_sh_bases=active)
        for _, eyes in reqs:
            probe.submit(sid, eyes)
            probe.drain(timeout_ms=30000)
            for c in probe.poll():
                probe.release(c.ticket)
        probe.submit(sid, reqs[big][1])
        probe.drain(timeout_ms=30000)
        one = probe.stats()["peak_resident_bytes"]
    budget = int(one * 1.15)
    with Server(DEV, max_in_flight=2, max_batch_requests=8, hbm_budget_bytes=budget) as srv:
        sid = srv.add_scene(*gt, K=8, active_sh_bases=active)
        srv.pause()
        for k, (_, eyes) in enumerate(reqs):
            srv.submit(sid, eyes, tag=k)
        srv.resume()
        got = {}
        while len(got) < len(reqs):
            cs = srv.poll(wait_ms=10000)
            assert cs
            for c in cs:
                assert c.ok, c.message
                got[c.tag] = tuple(x.clone() for x in c.images)
                srv.release(c.ticket)
        st = srv.stats()
    assert st["peak_resident_bytes"] <= budget
    assert st["max_frame_requests"] == 1  # two requests never fitted into one frame
    for k in range(len(reqs)):
        assert torch.equal(got[k][0], ref[k][0]) and torch.equal(got[k][1], ref[k][1])


def test_requests_that_cannot_fit_fail_cleanly(scenes):
    gt, active = scenes[0]
    scene_bytes = sum(t.numel() * t.element_size() for t in gt)
    with Server(DEV, hbm_budget_bytes=32 << 20) as srv:
        big = scene.make_gaussians(200000, 3, seed=4)
        bt = F.gaussians_to_torch(big, DEV)
        with pytest.raises(_lib.FhtgsError) as ei:
            srv.add_scene(*bt, K=8, active_sh_bases=16)  # 47 MB of Gaussians > 32 MB budget
        assert ei.value.status == 3
    # a budget that holds the scene but never a frame: the request fails with OUT_OF_MEMORY
    with Server(DEV, hbm_budget_bytes=scene_bytes + (4 << 20)) as srv:
        sid = srv.add_scene(*gt, K=8, active_sh_bases=active)
        srv.submit(sid, make_requests(1, 1)[0][1])
        cs = srv.poll(wait_ms=10000)
        assert len(cs) == 1 and cs[0].status == 3 and "budget" in cs[0].message
        assert srv.stats()["failed"] == 1


def test_overflowing_frame_is_rendered_again(scenes):
    """Gaussians that each cover the whole view overflow the first capacity estimate; the
    frame is rendered again with more room and equals the blocking path."""
    rng = np.random.default_rng(0)
    n = 20000
    g = scene.make_gaussians(n, 0, seed=8)
    # ~2.5-unit cutoff radius at 6 units: about 100 of the 300 tiles each, 2M+ instances per eye
    # against a first capacity of 2^20; the camera stays outside every cutoff ellipsoid
    g.positions[:] = rng.normal(0, 0.05, size=(n, 3)).astype(np.float32)
    g.scales[:] = 0.8
    gt = F.gaussians_to_torch(g, DEV)
    left, right = scene.make_stereo_views(320, 240)
    st = [F.settings_from_view(v, K=8, active_sh_bases=1, device=DEV) for v in (left, right)]
    a, b = F._C_stereo.render(*gt, *st[0].as_tuple(), *st[1].as_tuple(), True, False, False)
    with Server(DEV) as srv:
        sid = srv.add_scene(*gt, K=8, active_sh_bases=1)
        srv.submit(sid, [left, right])
        cs = srv.poll(wait_ms=30000)
        stats = srv.stats()
        assert len(cs) == 1 and cs[0].ok, cs[0].message if cs else "no completion"
        assert stats["retries"] >= 1
        assert torch.equal(cs[0].images[0], a) and torch.equal(cs[0].images[1], b)


def test_removed_scene_and_bad_requests(scenes):
    gt, active = scenes[2]
    with Server(DEV, max_in_flight=1) as srv:
        sid = srv.add_scene(*gt, K=8, active_sh_bases=active)
        eyes = make_requests(1, 1)[0][1]
        with pytest.raises(_lib.FhtgsError):
            srv.submit(sid + 7, eyes)
        with pytest.raises(ValueError):
            srv.submit(sid, eyes * 2)
        bad = F.settings_from_view(eyes[0], K=8, active_sh_bases=active, device=DEV)._replace(width=0)
        with pytest.raises(_lib.FhtgsError):
            srv.submit(sid, [bad])
        srv.remove_scene(sid)
        with pytest.raises(_lib.FhtgsError):
            srv.submit(sid, eyes)


def test_server_outputs_are_recycled(scenes):
    gt, active = scenes[2]
    reqs = make_requests(8, 1, seed=11)
    with Server(DEV, max_in_flight=1, max_batch_requests=1) as srv:
        sid = srv.add_scene(*gt, K=8, active_sh_bases=active)
        sizes = []
        for rnd in range(2):
            for k, (_, eyes) in enumerate(reqs):
                srv.submit(sid, eyes, tag=k)
                cs = srv.poll(wait_ms=10000)
                assert len(cs) == 1 and cs[0].ok
                srv.release(cs[0].ticket)
                sizes.append(srv.stats()["resident_bytes"])
        with pytest.raises(_lib.FhtgsError):
            srv.release(cs[0].ticket)  # released twice
    # the second round finds every output buffer and table in the pool: nothing new is held
    assert len(set(sizes[len(reqs):])) == 1 and sizes[-1] == sizes[len(reqs) - 1]


def test_ring_foveation_scenes_match_the_renderer(scenes):
    """A scene registered with ring foveation is served exactly as Renderer renders it."""
    gt, active = scenes[0]
    reqs = make_requests(4, 1, seed=21)
    r = F.Renderer(DEV)
    r.set_foveation("rings", 0.2, 0.5)
    ref = []
    for _, eyes in reqs:
        st = [F.settings_from_view(v, K=8, active_sh_bases=active, device=DEV) for v in eyes]
        ref.append([x.clone() for x in r.render(*gt, st, fast_math=True)])
    r.close()
    with Server(DEV, max_in_flight=2, max_batch_requests=4) as srv:
        sid = srv.add_scene(*gt, K=8, active_sh_bases=active, foveation="rings", rings=(0.2, 0.5))
        srv.pause()
        for k, (_, eyes) in enumerate(reqs):
            srv.submit(sid, eyes, tag=k)
        srv.resume()
        srv.drain(timeout_ms=30000)
        comps = srv.poll()
        assert len(comps) == len(reqs) and all(c.ok for c in comps)
        for c in comps:
            for e in range(2):
                assert torch.equal(c.images[e], ref[c.tag][e]), f"request {c.tag} eye {e}"


def test_destroy_with_frames_in_flight_returns(scenes):
    """Closing a server while its frames run: the running frames finish, queued requests are
    dropped, and the call returns (the scheduler waits for the frames' completion callbacks with
    its lock released; it once spun holding the lock those callbacks need)."""
    import threading
    import time

    reqs = make_requests(16, len(scenes), seed=21)
    srv = Server(DEV, max_in_flight=2, max_batch_requests=2)
    ids = add_all(srv, scenes)
    for k, (si, eyes) in enumerate(reqs):
        srv.submit(ids[si], eyes, tag=k)
    time.sleep(0.005)  # the first frames are on the GPU, the rest queued
    t = threading.Thread(target=srv.close, daemon=True)
    t0 = time.perf_counter()
    t.start()
    t.join(30.0)
    assert not t.is_alive(), "fhtgs_server_destroy did not return within 30 s"
    assert time.perf_counter() - t0 < 30.0
    torch.cuda.synchronize()
