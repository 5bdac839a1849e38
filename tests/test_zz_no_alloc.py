"""GPU test of fhtgs_sort_instances_noalloc, the instance sort that allocates no device memory.

Some callers of this library cannot allocate: a VR compositor or display thread with a hard
frame deadline (a cudaMalloc/cudaFree can synchronise the device and stall it), or a plugin
whose host application owns the device-memory budget.  They call the renderer's stable
instance sort with their own input and output buffers, and its working memory is a fixed array
inside libfhtgs.so.  This test calls that entry point through the C ABI and checks that its
output equals the sorted instances produced by the existing entry point
(fhtgs_render_views_sync, read back with fhtgs_copy_intermediates) — bit-exact, as for all
integer outputs — on two calls in a row with different data, sizes and key widths, so that
contents the shared scratch array kept from the first call would show up in the second.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import foveatedhtgscudabackend_b200 as F
from foveatedhtgscudabackend_b200 import _lib, scene

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def sorted_instances_from_renderer(n, sh_degree, seed, w, h):
    """Sorted (key, value) pairs of one view from the existing rendering entry point."""
    g = scene.make_gaussians(n, sh_degree, seed=seed)
    v = scene.make_view(w, h, gaze_ndc=(0.25, -0.2))
    r = F.Renderer("cuda:0")
    try:
        r.render(*F.gaussians_to_torch(g), [F.settings_from_view(v, K=8, active_sh_bases=(sh_degree + 1) ** 2)])
        m = r.intermediates(0)
    finally:
        r.close()
    end_bit = m["end_bit"]
    key_dtype = np.uint16 if end_bit <= 16 else np.uint32
    keys = m["keys"].astype(key_dtype)
    vals = m["values"].astype(np.uint32)
    assert 0 < keys.size <= MAX_PAIRS
    # The instances in the order they are emitted (primitive, then tile order; the sentinels of
    # over-counted slots close each primitive's run): a lexicographic sort by (value, key).
    order = np.lexsort((keys, vals))
    return keys[order], vals[order], keys, vals, end_bit


def noalloc_sort(keys_in: np.ndarray, vals_in: np.ndarray, end_bit: int, in_place: bool = False):
    lib = _lib.load()
    dev = torch.device("cuda:0")
    k_in = torch.from_numpy(keys_in).to(dev)
    v_in = torch.from_numpy(vals_in).to(dev)
    k_out = k_in if in_place else torch.empty_like(k_in)
    v_out = v_in if in_place else torch.empty_like(v_in)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib.fhtgs_sort_instances_noalloc(k_in.data_ptr(), v_in.data_ptr(), k_out.data_ptr(), v_out.data_ptr(),
                                          int(keys_in.size), int(keys_in.itemsize), int(end_bit), stream)
    _lib.check(st)
    torch.cuda.synchronize(dev)
    out = (k_out.cpu().numpy(), v_out.cpu().numpy())
    if not in_place:  # the inputs are left as they were
        assert np.array_equal(k_in.cpu().numpy(), keys_in) and np.array_equal(v_in.cpu().numpy(), vals_in)
    return out


def test_noalloc_sort_matches_renderer_on_two_calls_in_a_row():
    # call 1: 16-bit keys (640x480 grid, 13 key bits); call 2: 32-bit keys (2064x2208, 17 bits)
    a = sorted_instances_from_renderer(30000, 3, 1, 640, 480)
    b = sorted_instances_from_renderer(6000, 0, 2, 2064, 2208)
    assert a[0].dtype == np.uint16 and b[0].dtype == np.uint32
    for keys_in, vals_in, keys_ref, vals_ref, end_bit in (a, b):
        keys, vals = noalloc_sort(keys_in, vals_in, end_bit)
        assert np.array_equal(keys, keys_ref)
        assert np.array_equal(vals, vals_ref)


def test_noalloc_sort_rejects_sizes_beyond_its_maximum():
    lib = _lib.load()
    st = lib.fhtgs_sort_instances_noalloc(None, None, None, None, MAX_PAIRS + 1, 4, 17, None)
    assert st == 1
    assert b"1048576" in lib.fhtgs_last_error()


def test_noalloc_sort_orders_by_the_bits_below_end_bit_only():
    """Keys with bits set at and above end_bit (end_bit not a multiple of 8): the order is the
    stable order of the low end_bit bits, and every key comes out with all its bits."""
    rng = np.random.default_rng(7)
    for dtype, end_bit, n in ((np.uint16, 11, 70_000), (np.uint32, 17, 300_001), (np.uint32, 20, 4097)):
        keys = rng.integers(0, np.iinfo(dtype).max, size=n, dtype=np.uint64).astype(dtype)
        vals = rng.permutation(n).astype(np.uint32)
        order = np.argsort(keys.astype(np.uint64) & ((1 << end_bit) - 1), kind="stable")
        got_k, got_v = noalloc_sort(keys, vals, end_bit)
        assert np.array_equal(got_k, keys[order]), f"{dtype.__name__} end_bit {end_bit}"
        assert np.array_equal(got_v, vals[order]), f"{dtype.__name__} end_bit {end_bit}"


def test_noalloc_sort_in_place_equals_out_of_place():
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 13, size=200_000, dtype=np.uint16)
    vals = np.arange(keys.size, dtype=np.uint32)
    ref = noalloc_sort(keys, vals, 13)
    got = noalloc_sort(keys, vals, 13, in_place=True)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
