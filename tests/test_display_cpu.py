"""CPU checks of the overlay / tile-mask / display-packing restatement and of the host-side argument
handling of their C-ABI entry points (no device work).

The overlay restatement (oracle/display_oracle.py) is pinned against images written by the
reference's own `_C_visualization` module (tests/golden/visualization/, made by
tests/golden/make_golden_visualization.py): bit-exact, every case.
"""
import os

import numpy as np
import pytest

import display_oracle as D
from foveatedhtgscudabackend_b200 import _lib, scene
from golden.make_golden_visualization import GREY, ORACLE_ONLY_TILE_CASES, all_cases, case_inputs

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "visualization", "reference_overlays.npz")


def run_oracle(name: str) -> np.ndarray:
    img, kind, a = case_inputs(name)
    if kind == "gaze":
        return D.visualize_gaze(img, a["gaze"], a["color"], a["size"], a["vtype"], a["to_chw"])
    return D.visualize_tile_boundaries(img, a["mask"], a["gaze"], a["to_chw"])


@pytest.fixture(scope="module")
def reference_overlays():
    if not os.path.exists(FIXTURE):
        pytest.fail(f"{FIXTURE} missing; regenerate it with tests/golden/make_golden_visualization.py")
    return dict(np.load(FIXTURE))


@pytest.mark.parametrize("name", all_cases())
def test_overlay_restatement_matches_reference_images(reference_overlays, name):
    ref = reference_overlays[name]
    out = run_oracle(name)
    assert out.shape == ref.shape
    assert np.array_equal(out, ref), f"{name}: {int(np.sum(out != ref))} values differ"


def test_golden_overlays_cover_every_class_and_marker(reference_overlays):
    colors = {tuple(c) for c in (D.ORANGE, D.LIGHT_BLUE, D.GREEN)}
    img = reference_overlays["tiles_all_center"]
    seen = {tuple(img[:, y, x]) for y, x in zip(*np.nonzero(np.any(img != GREY, axis=0)))}
    assert colors <= seen
    assert not np.any(reference_overlays["tiles_single_periphery"] != GREY)  # one entry: nothing drawn
    assert np.any(reference_overlays["tiles_single_fovea"] != GREY)  # one fovea tile = 4 entries


def test_no_visible_tile_draws_nothing():
    for name in ORACLE_ONLY_TILE_CASES:
        img = run_oracle(name)
        assert np.all(img == GREY)


@pytest.mark.parametrize("w,h,vis", [(2064, 2208, None), (640, 480, "random"), (16, 16, None), (1, 1, None),
                                     (513, 1, "random"), (16 * 32, 16, "lens"), (1003, 757, "lens")])
def test_tile_mask_restatement_matches_scene_tables(w, h, vis):
    gw, gh = -(-w // 16), -(-h // 16)
    visible = None
    if vis == "random":
        visible = scene.random_visibility(gw, gh, 0.6, 7)
    elif vis == "lens":
        visible = scene.lens_visibility(gw, gh)
    words, sat, fov = D.tile_masks(w, h, visible)
    s_words, s_sat = scene.visibility_tables(gw, gh, visible)
    assert np.array_equal(words, s_words) and np.array_equal(sat, s_sat)
    assert np.array_equal(fov, scene.fovea_table())


def test_pack_restatement_rounding_and_layout():
    a = np.array([[[0.0, 0.6 / 255, 1.6 / 255], [1.0, 2.0, -1.0], [np.nan, 0.998, 0.5]]], np.float32)  # HWC 1x3
    b = np.zeros_like(a)
    out = D.pack_display([a, b], to_chw=False)
    assert out.shape == (1, 6, 4) and out.dtype == np.uint8
    assert list(out[0, 0]) == [0, 1, 2, 255]
    assert list(out[0, 1]) == [255, 255, 0, 255]
    assert list(out[0, 2]) == [0, 254, 128, 255]
    assert np.all(out[0, 3:, :3] == 0) and np.all(out[0, :, 3] == 255)
    bgra = D.pack_display([np.transpose(a, (2, 0, 1))], to_chw=True, bgra=True)
    assert np.array_equal(bgra[..., :3], out[:, :3, 2::-1])


def test_entry_points_reject_bad_arguments_without_device_work():
    lib = _lib.load()
    assert lib.fhtgs_build_tile_masks(None, 0, 10, None, None, None, None) == 1
    assert lib.fhtgs_build_tile_masks(None, 10, 10, None, None, None, None) == 1
    assert lib.fhtgs_pack_display(None, 1, 4, 4, 1, 0, None, None) == 1
    assert lib.fhtgs_visualize_gaze(None, 4, 4, 0.0, 0.0, 1.0, 1.0, 1.0, 0, 4, 1, None) == 1
    assert lib.fhtgs_visualize_gaze(1, 4, 4, 0.0, 0.0, 1.0, 1.0, 1.0, 256, 4, 1, None) == 1
    assert b"8 bits" in lib.fhtgs_last_error()
    assert lib.fhtgs_visualize_tile_boundaries(None, 4, 4, None, 0.0, 0.0, 1, None) == 1
