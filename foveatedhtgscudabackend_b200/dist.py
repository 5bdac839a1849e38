"""Multi-GPU plumbing: one process per GPU, the scene replicated, views sharded.

Views are independent once their camera is known, and the K-buffer blend is not associative
over a split of the Gaussians, so the renderer scales by giving each rank its own views (or
frames) of a replicated scene.  Nothing crosses NVLink on the data path; torch.distributed is
used for the barrier and for taking the maximum of the per-rank device times.
"""
from __future__ import annotations

import datetime
import os
import socket
import subprocess
import sys


def world() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def free_port() -> int:
    """A TCP port on 127.0.0.1 that nothing listens on right now."""
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return int(s.getsockname()[1])


def launch_ranks(n: int, argv: list[str], port: int | None = None, extra_env: dict | None = None) -> int:
    """Runs `python argv...` as n ranks of one node under torch.distributed.run (rendezvous on
    127.0.0.1, one process per GPU) and returns the launcher's exit status.  NCCL's
    initialisation log (one line per rank and communicator, with its rank count) goes to
    stderr unless the caller configured NCCL logging."""
    env = dict(os.environ)
    env.update(extra_env or {})
    env.setdefault("NCCL_DEBUG", "INFO")
    env.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    env.setdefault("NCCL_DEBUG_FILE", "/dev/stderr")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port or free_port())] + list(argv)
    return subprocess.call(cmd, env=env)


def init(backend: str | None = None, timeout_s: float = 300.0) -> tuple[int, int, int]:
    """Initialises the process group when WORLD_SIZE > 1 (NCCL on GPUs, gloo otherwise)."""
    import torch
    import torch.distributed as dist
    n, rank, local = world()
    if n > 1 and not dist.is_initialized():
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
            # NCCL's initialisation log (rank counts) on stderr, unless configured otherwise
            os.environ.setdefault("NCCL_DEBUG", "INFO")
            os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
            os.environ.setdefault("NCCL_DEBUG_FILE", "/dev/stderr")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return n, rank, local


def shard(n_items: int, n_ranks: int, rank: int) -> list[int]:
    """Contiguous, balanced share of n_items for `rank` (sizes differ by at most one)."""
    base, extra = divmod(n_items, n_ranks)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def max_over_ranks(x: float) -> float:
    """Maximum of a per-rank value (e.g. device milliseconds) over all ranks."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def finalize() -> None:
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()
