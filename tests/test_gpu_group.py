"""GPU tests of the replica group (fhtgs_server_group_*): scenes replicated peer to peer, each
request routed whole to one replica, completions merged.

This pool gives one GPU, so the group here holds two replicas on device 0: the first borrows
the caller's arrays, the second renders from its own copy made by cudaMemcpyPeerAsync (within
one device), so the replication, the routing and the merged polling all run; the same code with
distinct device ids places the replicas on distinct GPUs.

Tolerance: none.  Every request's images must equal, bit for bit, the drop-in `_C_stereo.render`
of the same views alone, whichever replica rendered them (max-abs 2e-3 and
PSNR >= 50 dB; replication copies the scene exactly, so the test asks for equality).
"""
import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import scene
from foveatedhtgscudabackend_b200.serving import ServerGroup

from test_gpu_serving import make_requests, render_reference

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def scenes():
    out = []
    for n, seed, deg in ((30000, 1, 3), (15000, 3, 0)):
        g = scene.make_gaussians(n, deg, seed=seed)
        out.append((F.gaussians_to_torch(g, DEV), (deg + 1) ** 2))
    return out


def test_group_serves_every_request_once_exactly_and_balanced(scenes):
    reqs = make_requests(24, len(scenes), seed=11)
    ref = render_reference(scenes, reqs)
    with ServerGroup([0, 0], hbm_budget_bytes=20e9, max_in_flight=2, max_batch_requests=4) as grp:
        ids = [grp.add_scene(*gt, K=8, active_sh_bases=active) for gt, active in scenes]
        routed = {}
        for k, (si, eyes) in enumerate(reqs):
            ticket, replica = grp.submit(ids[si], eyes, tag=k)
            assert ticket not in routed
            routed[ticket] = replica
        got, seen = {}, set()
        while len(got) < len(reqs):
            cs = grp.poll(wait_ms=5000)
            assert cs, "no completion within 5 s"
            for c in cs:
                assert c.ok, c.message
                assert c.ticket in routed and c.ticket not in seen   # every request completes once
                seen.add(c.ticket)
                assert c.replica == routed[c.ticket] and c.device == 0
                got[c.tag] = tuple(x.clone() for x in c.images)
                grp.release(c.ticket)
        grp.drain(10000)
        per = [grp.stats(r) for r in range(2)]
    for k in range(len(reqs)):
        for a, b in zip(got[k], ref[k]):
            assert torch.equal(a, b), f"request {k} differs from the request rendered alone"
    counts = [p["submitted"] for p in per]
    assert sum(counts) == len(reqs) and min(counts) >= len(reqs) // 4   # both replicas served
    assert all(p["completed"] == p["submitted"] and p["outstanding_cost"] == 0 for p in per)


def test_requests_with_device_buffers_stay_on_their_device(scenes):
    (gt, active), = scenes[:1]
    reqs = make_requests(4, 1, seed=12)
    ref = render_reference(scenes[:1], reqs)
    with ServerGroup([0, 0], hbm_budget_bytes=20e9) as grp:
        sid = grp.add_scene(*gt, K=8, active_sh_bases=active)
        out = []
        for k, (_, eyes) in enumerate(reqs):
            imgs = [torch.zeros((3, v.height, v.width), device=DEV) for v in eyes]
            ticket, replica = grp.submit(sid, eyes, images=imgs, tag=k)
            assert 0 <= replica < 2
            out.append(imgs)
        n = 0
        while n < len(reqs):
            cs = grp.poll(wait_ms=5000)
            assert cs
            for c in cs:
                assert c.ok, c.message
                n += 1
        torch.cuda.synchronize()
    for k in range(len(reqs)):
        for a, b in zip(out[k], ref[k]):
            assert torch.equal(a, b)


def test_group_rejects_bad_arguments(scenes):
    with pytest.raises(F.FhtgsError):
        ServerGroup([], hbm_budget_bytes=1e9)
    with pytest.raises(F.FhtgsError):
        ServerGroup([0, 99], hbm_budget_bytes=1e9)   # no such device: nothing leaks
    with ServerGroup([0], hbm_budget_bytes=20e9) as grp:
        with pytest.raises(F.FhtgsError):
            grp.release(12345)
