"""The C-ABI library loads and exports every entry point include/fhtgs.h declares (no GPU calls)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from foveatedhtgscudabackend_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fhtgs.h")


def declared_functions() -> list[str]:
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fhtgs_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for must in ("fhtgs_render_mono", "fhtgs_benchmark_mono", "fhtgs_render_stereo", "fhtgs_render_views",
                 "fhtgs_render_views_sync", "fhtgs_context_create", "fhtgs_context_destroy", "fhtgs_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s+(fhtgs_[a-z0-9_]+)", out))
    for name in declared_functions():
        assert name in exported, f"{name} declared in fhtgs.h but not exported"
        assert hasattr(lib, name)
    assert set(_lib.SIGNATURES) == set(declared_functions())


def test_abi_version_and_error_paths_without_device_work():
    lib = _lib.load()
    assert lib.fhtgs_abi_version() == 2
    assert lib.fhtgs_render_views(None, None, None, 0, None, None) == 1  # invalid argument
    assert b"null" in lib.fhtgs_last_error()
    fi = _lib.FrameInfo()
    assert lib.fhtgs_get_frame_info(None, 0, C.byref(fi)) == 1
    assert lib.fhtgs_context_destroy(None) == 0


def test_library_has_no_torch_or_python_dependency():
    out = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "torch" not in out and "python" not in out and "libc10" not in out


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(_lib.FhtgsError):
        _lib.load(str(tmp_path / "nope.so"))
