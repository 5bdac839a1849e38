"""Builds libfhtgs.so (sm_100a) in-tree with nvcc.

    python -m foveatedhtgscudabackend_b200.build [--force] [--jobs N]

Translation units:
  csrc/kernels_fast.cu  -use_fast_math  (arithmetic of the reference's _C_benchmarking / _C_stereo)
  csrc/kernels_ieee.cu  IEEE            (arithmetic of the reference's _C)
  csrc/fhtgs_host.cu    context, arena, orchestration, C ABI (include/fhtgs.h)
  csrc/fhtgs_noalloc.cu the instance sort with a static working array
  csrc/fhtgs_extras.cu  tile-mask builder, display packing, debug overlays
  csrc/fhtgs_server.cu  request server: resident scenes, continuous batching, HBM admission
  csrc/fhtgs_group.cu   replica group of servers over several devices (routing: fhtgs_route.h)
The CUDA runtime is linked statically; the library has no torch dependency.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "lib")
OBJ_DIR = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(OUT_DIR, "libfhtgs.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
UNITS = [
    ("kernels_fast.cu", ["-use_fast_math"]),
    ("kernels_ieee.cu", []),
    ("fhtgs_host.cu", []),
    ("fhtgs_noalloc.cu", []),
    ("fhtgs_extras.cu", []),
    ("fhtgs_server.cu", []),
    ("fhtgs_group.cu", []),
]
HEADERS = ["fhtgs_types.cuh", "fhtgs_math.cuh", "fhtgs_kernels.cuh", "fhtgs_internal.h", "fhtgs_route.h"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; libfhtgs needs the CUDA toolkit to build")


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def _compile(src: str, extra: list[str], force: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "fhtgs.h"), os.path.abspath(__file__)]
    if not force and _mtime(obj) >= max(_mtime(d) for d in deps):
        return obj
    cmd = [nvcc()] + ARCH + COMMON + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 3) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        objs = list(ex.map(lambda u: _compile(u[0], u[1], force), UNITS))
    if force or _mtime(LIB) < max(_mtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-fPIC"] + objs + ["-o", tmp]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=3)
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs))
    return 0


if __name__ == "__main__":
    sys.exit(main())
