"""Shared test helpers: image metrics, golden-case loading, integer-parity comparisons."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Image tolerances against the reference (north star): max-abs 2e-3 and PSNR >= 50 dB.
REF_MAX_ABS = 2e-3
REF_PSNR_DB = 50.0


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(1.0 / mse)


def max_abs(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)))) if np.size(a) else 0.0


def golden_cases() -> list[str]:
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name: str) -> tuple[dict, dict]:
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        case = json.load(f)
    data = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    return case, data


def view_data(data: dict, i: int) -> dict:
    p = f"v{i}_"
    return {k[len(p):]: v for k, v in data.items() if k.startswith(p)}


def sentinel_for(end_bit: int) -> int:
    return 0xFFFF if end_bit <= 16 else 0xFFFFFFFF


def assert_instances_equal(mine: dict, ref: dict, end_bit: int, what: str = ""):
    """Bit-exact comparison of instance count, sorted keys, sorted values (non-sentinel) and ranges."""
    m_ref = int(ref["n_instances"])
    assert int(mine["n_instances"]) == m_ref, f"{what}: M {mine['n_instances']} != {m_ref}"
    k_ref = np.asarray(ref["keys"], np.uint32)[:m_ref]
    k_me = np.asarray(mine["keys"], np.uint32)[:m_ref]
    assert np.array_equal(k_me, k_ref), f"{what}: sorted keys differ at {np.flatnonzero(k_me != k_ref)[:10]}"
    valid = k_ref != sentinel_for(end_bit)
    v_ref = np.asarray(ref["values"], np.uint32)[:m_ref][valid]
    v_me = np.asarray(mine["values"], np.uint32)[:m_ref][valid]
    assert np.array_equal(v_me, v_ref), f"{what}: sorted values differ at {np.flatnonzero(v_me != v_ref)[:10]}"
    r_ref = np.asarray(ref["instance_ranges"], np.uint32).reshape(-1, 2)
    r_me = np.asarray(mine["instance_ranges"], np.uint32).reshape(-1, 2)
    assert np.array_equal(r_me, r_ref), f"{what}: tile ranges differ for tiles {np.flatnonzero((r_me != r_ref).any(1))[:10]}"


def assert_tiles_equal(mine: dict, ref: dict, what: str = ""):
    na = int(ref["n_active_tiles"])
    assert int(mine["n_active_tiles"]) == na, f"{what}: active tiles {mine['n_active_tiles']} != {na}"
    assert np.array_equal(np.asarray(mine["tile_index_map_partitioned"])[:na],
                          np.asarray(ref["tile_index_map_partitioned"])[:na]), f"{what}: tile map differs"
    assert np.array_equal(np.asarray(mine["tile_type_partitioned"])[:na],
                          np.asarray(ref["tile_type_partitioned"])[:na]), f"{what}: tile types differ"
    assert np.array_equal(np.asarray(mine["partition_ranges"], np.uint32).reshape(-1),
                          np.asarray(ref["partition_ranges"], np.uint32).reshape(-1)), f"{what}: partition ranges differ"
