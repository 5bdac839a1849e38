"""Routing policy of the replica group (csrc/fhtgs_route.h), compiled with g++ alone and driven
from a simulated request stream: every request goes to exactly one eligible replica, requests
bound to a device stay on it, equal loads alternate round robin, and the outstanding work of
the replicas stays balanced under a stream of uneven requests."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "foveatedhtgscudabackend_b200", "csrc")

WRAPPER = r"""
#include <vector>
#include "fhtgs_route.h"
extern "C" int route_pick(const int* devices, const long long* costs, int n, int device, unsigned long long* cursor) {
    std::vector<fhtgs::ReplicaLoad> r(n);
    for (int i = 0; i < n; ++i) r[i] = fhtgs::ReplicaLoad{devices[i], costs[i]};
    uint64_t c = *cursor;
    const int k = fhtgs::pick_replica(r.data(), n, device, &c);
    *cursor = c;
    return k;
}
extern "C" long long route_cost(const long long* px, int n_eyes, long long n_gaussians) {
    const int64_t p[2] = {px[0], n_eyes > 1 ? px[1] : 0};
    return fhtgs::request_cost(p, n_eyes, n_gaussians);
}
"""


@pytest.fixture(scope="module")
def route(tmp_path_factory):
    d = tmp_path_factory.mktemp("route")
    src = d / "route.cpp"
    src.write_text(WRAPPER)
    so = d / "libroute.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I" + CSRC, str(src), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))
    lib.route_pick.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.c_int, C.c_int,
                               C.POINTER(C.c_ulonglong)]
    lib.route_pick.restype = C.c_int
    lib.route_cost.argtypes = [C.POINTER(C.c_longlong), C.c_int, C.c_longlong]
    lib.route_cost.restype = C.c_longlong
    return lib


class Group:
    def __init__(self, lib, devices):
        self.lib = lib
        self.devices = list(devices)
        self.load = [0] * len(devices)
        self.cursor = C.c_ulonglong(0)

    def pick(self, device=-1):
        n = len(self.devices)
        d = (C.c_int * n)(*self.devices)
        c = (C.c_longlong * n)(*self.load)
        return self.lib.route_pick(d, c, n, device, C.byref(self.cursor))


def test_equal_loads_alternate_round_robin(route):
    g = Group(route, [0, 1, 2, 3])
    assert [g.pick() for _ in range(8)] == [0, 1, 2, 3, 0, 1, 2, 3]


def test_requests_bound_to_a_device_stay_on_it(route):
    g = Group(route, [0, 1, 1, 2])
    for _ in range(20):
        k = g.pick(device=1)
        assert g.devices[k] == 1
        g.load[k] += 10
    assert g.load[1] == g.load[2] == 100  # the two replicas of device 1 share the work
    assert g.pick(device=5) == -1          # no replica there


def test_cost_grows_with_pixels_and_gaussians(route):
    px = (C.c_longlong * 2)(2064 * 2208, 2064 * 2208)
    stereo_big = route.route_cost(px, 2, 4_000_000)
    mono_big = route.route_cost(px, 1, 4_000_000)
    stereo_small = route.route_cost(px, 2, 500_000)
    assert stereo_big == 2 * mono_big and stereo_big > stereo_small > 0


def _stream(route, g, n, rate, rng):
    """n stereo requests over 3 scenes and 2 resolutions; every replica completes `rate` units of
    work per arrival.  Returns the routed replica per request, the work routed to each replica,
    the largest request cost and the largest spread of outstanding work seen after a routing."""
    scenes = (500_000, 2_000_000, 4_000_000)
    sizes = ((1440, 1584), (2064, 2208))
    routed, total, spread, max_cost = [], [0] * len(g.devices), 0, 0
    for _ in range(n):
        w, h = sizes[rng.integers(2)]
        px = (C.c_longlong * 2)(w * h, w * h)
        cost = route.route_cost(px, 2, scenes[rng.integers(3)])
        max_cost = max(max_cost, cost)
        k = g.pick()
        assert 0 <= k < len(g.devices)
        routed.append(k)
        g.load[k] += cost
        total[k] += cost
        spread = max(spread, max(g.load) - min(g.load))
        g.load = [max(0, int(x - rate)) for x in g.load]
    return routed, total, max_cost, spread


def test_uneven_stream_every_request_served_once_and_balanced(route):
    """Each request is routed to exactly one replica; the outstanding work of the replicas never
    spreads by more than one request's cost; and when the replicas are kept busy, the work each
    received over the whole stream differs by no more than a few requests."""
    rng = np.random.default_rng(0)
    g = Group(route, list(range(8)))
    mean_cost = 6.9e6 * 9.3  # mean pixels of a stereo request x mean scene factor
    routed, total, max_cost, spread = _stream(route, g, 5000, 0.9 * mean_cost / 8, rng)  # overloaded
    assert len(routed) == 5000 and sorted(set(routed)) == list(range(8))
    assert spread <= max_cost
    assert max(total) - min(total) <= 2 * max_cost
    # lightly loaded: queues run empty, yet the outstanding spread stays within one request
    g2 = Group(route, list(range(8)))
    _, _, max_cost2, spread2 = _stream(route, g2, 5000, 3.0 * mean_cost / 8, rng)
    assert spread2 <= max_cost2
