"""Multi-rank host logic on CPU with gloo (world size 2): view sharding and max-over-ranks timing."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from foveatedhtgscudabackend_b200 import dist as D


def test_shard_covers_items_once_and_balanced():
    for n in (0, 1, 2, 7, 64, 65):
        for world in (1, 2, 3, 8):
            parts = [D.shard(n, world, r) for r in range(world)]
            flat = [i for p in parts for i in p]
            assert flat == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    n, r, _ = D.init(backend="gloo", timeout_s=60)
    try:
        mine = D.shard(10, n, r)
        t = 5.0 + 3.0 * r  # a per-rank "device time"
        D.barrier()
        out[r] = (n, r, mine, D.max_over_ranks(t))
    finally:
        D.finalize()


@pytest.mark.timeout(120)
def test_two_ranks_gloo_shard_and_max():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert res[0][0] == 2 and res[1][0] == 2
    assert res[0][2] + res[1][2] == list(range(10))
    assert res[0][3] == res[1][3] == 8.0


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.timeout(300)
def test_bench_gpus_2_starts_two_ranks_and_prints_one_line(tmp_path):
    """`bench.py --gpus 2` outside a launcher starts two ranks itself (torchrun on 127.0.0.1);
    rank 0 prints the only JSON line, with n_gpus = 2.  On CPU the reference arm is the one that
    runs (the host-core restatement; its CUDA leg reports no device), here on a tiny scene."""
    import json
    import subprocess
    import sys
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--n-gaussians",
           "3000", "--width", "96", "--height", "80", "--sh-degree", "1", "--steps", "1", "--warmup", "0",
           "--cpu-budget-s", "5"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=280, env=env, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["n_gpus"] == 2 and line["impl"] == "reference"
    assert "unavailable" in line["reference_cuda"]


@pytest.mark.timeout(120)
def test_bench_refuses_a_world_that_differs_from_gpus(tmp_path):
    import subprocess
    import sys
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, timeout=100, env=env, cwd=str(tmp_path))
    assert r.returncode != 0 and "--gpus 2 but 1 rank" in r.stderr
