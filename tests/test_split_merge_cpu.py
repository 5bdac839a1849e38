"""CPU check of the split blend's merge rule (no GPU): a pixel's fragment stream blended serially
with the K-buffer of blend_cu (reference inference.cuh:188-240) against the same stream cut into
contiguous segments, each walked from an empty K-buffer that records the fragments entering it,
then merged by replaying the records in order from the first segment's state.

The K-buffer contents must agree exactly (same insertions and evictions, so the same RGBA8
colours); the tail sum and its transmittance agree to float32 rounding.  The exact split (every
segment logs its pairs, the merge replays all logs in order) must agree bit for bit.
"""
import numpy as np
import pytest

MIN_ALPHA, MIN_CORE = np.float32(1 / 255), np.float32(1 / 20)
BIG = np.float32(3.402823466e38)


def pack(pm):
    q = np.floor(np.clip(pm, 0, 1) * np.float32(255) + np.float32(0.5)).astype(np.uint32)
    return int(q[0] | (q[1] << 8) | (q[2] << 16) | (q[3] << 24))


def unpack(c):
    return np.array([(c >> s) & 0xFF for s in (0, 8, 16, 24)], np.float32) / np.float32(255)


def insert(core, depth, color):
    """Inserts (depth, color) if closer than the K-th; returns the evicted entry or None."""
    if not depth < core[-1][0]:
        return None
    f = (depth, color)
    for k in range(len(core)):
        if f[0] < core[k][0]:
            core[k], f = f, core[k]
    return f


def serial(frags, K):
    core = [(BIG, 0)] * K
    tail, T = np.zeros(4, np.float32), np.float32(1)
    for depth, pm in frags:
        if pm[3] < MIN_ALPHA:
            continue
        if pm[3] >= MIN_CORE:
            ev = insert(core, depth, pack(pm))
            if ev is not None:
                pm = unpack(ev[1])
        tail = tail + pm
        T = T * (np.float32(1) - pm[3])
    return core, tail, T


def segment(frags, K):
    """A later segment: empty K-buffer, fragments that enter it are recorded, not blended."""
    core = [(BIG, 0)] * K
    recs, tail, T = [], np.zeros(4, np.float32), np.float32(1)
    for depth, pm in frags:
        if pm[3] < MIN_ALPHA:
            continue
        if pm[3] >= MIN_CORE and insert(core, depth, pack(pm)) is not None:
            recs.append((depth, pm))
            continue
        tail = tail + pm
        T = T * (np.float32(1) - pm[3])
    return recs, tail, T


def split(frags, K, cuts):
    parts = np.split(np.arange(len(frags)), cuts)
    core, tail, T = serial([frags[i] for i in parts[0]], K)
    for p in parts[1:]:
        recs, t, tt = segment([frags[i] for i in p], K)
        tail, T = tail + t, T * tt
        for depth, pm in recs:
            ev = insert(core, depth, pack(pm))
            if ev is not None:
                pm = unpack(ev[1])
            tail = tail + pm
            T = T * (np.float32(1) - pm[3])
    return core, tail, T


def stream(rng, n, sorted_depth):
    depth = rng.uniform(1, 10, n).astype(np.float32)
    if sorted_depth:  # list order roughly follows depth, as the renderer's does
        depth = np.sort(depth) + rng.normal(0, 0.3, n).astype(np.float32)
    alpha = np.where(rng.random(n) < 0.3, rng.uniform(0, 0.06, n), rng.uniform(0, 0.99, n)).astype(np.float32)
    rgb = rng.random((n, 3)).astype(np.float32)
    return [(np.float32(d), np.append(c * a, a).astype(np.float32)) for d, c, a in zip(depth, rgb, alpha)]


@pytest.mark.parametrize("K", [1, 4, 8, 32])
@pytest.mark.parametrize("sorted_depth", [True, False])
def test_segmented_merge_reproduces_serial_k_buffer(K, sorted_depth):
    rng = np.random.default_rng(K * 7 + sorted_depth)
    for trial in range(20):
        n = int(rng.integers(1, 400))
        frags = stream(rng, n, sorted_depth)
        S = int(rng.integers(2, 9))
        cuts = sorted(int(c) for c in rng.integers(0, n + 1, S - 1))
        c0, t0, T0 = serial(frags, K)
        c1, t1, T1 = split(frags, K, cuts)
        assert c0 == c1, f"K-buffer differs (trial {trial})"
        np.testing.assert_allclose(t1, t0, rtol=2e-5, atol=1e-5)
        np.testing.assert_allclose(T1, T0, rtol=2e-5, atol=1e-6)


def test_ties_keep_list_order():
    # equal depths: the earlier fragment stays ahead, in both walks
    frags = [(np.float32(2.0), np.array([0.1, 0, 0, 0.5], np.float32)),
             (np.float32(2.0), np.array([0, 0.1, 0, 0.5], np.float32)),
             (np.float32(1.0), np.array([0, 0, 0.1, 0.5], np.float32))]
    assert serial(frags, 2)[0] == split(frags, 2, [1])[0] == split(frags, 2, [2])[0]


def exact_split(frags, K, cuts):
    """The exact split: each segment logs its pairs (alpha, or -1 where the pair is no fragment;
    depth) without a K-buffer, and the merge replays the logs of all segments in order with the
    walk's own steps."""
    log = []
    for p in np.split(np.arange(len(frags)), cuts):
        for i in p:
            depth, pm = frags[i]
            a = pm[3] if not pm[3] < MIN_ALPHA else np.float32(-1)
            log.append((depth, a, pm))
    core = [(BIG, 0)] * K
    tail, T = np.zeros(4, np.float32), np.float32(1)
    for depth, a, pm in log:
        if a < 0:
            continue
        if a >= MIN_CORE:
            ev = insert(core, depth, pack(pm))
            if ev is not None:
                pm = unpack(ev[1])
        tail = tail + pm
        T = T * (np.float32(1) - pm[3])
    return core, tail, T


@pytest.mark.parametrize("K", [1, 8, 32])
def test_exact_split_replay_is_the_serial_walk(K):
    rng = np.random.default_rng(100 + K)
    for trial in range(10):
        n = int(rng.integers(1, 300))
        frags = stream(rng, n, bool(trial % 2))
        cuts = sorted(int(c) for c in rng.integers(0, n + 1, int(rng.integers(1, 8))))
        c0, t0, T0 = serial(frags, K)
        c1, t1, T1 = exact_split(frags, K, cuts)
        assert c0 == c1
        assert np.array_equal(t0, t1) and T0 == T1  # same operations in the same order: bit for bit
