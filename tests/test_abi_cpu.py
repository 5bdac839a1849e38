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
    assert lib.fhtgs_abi_version() == 4
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


def test_struct_layouts_match_the_header(tmp_path):
    """ctypes mirrors of the C structs have the header's sizes and field offsets (gcc build)."""
    structs = {"fhtgs_primitives": _lib.Primitives, "fhtgs_view": _lib.View, "fhtgs_settings": _lib.Settings,
               "fhtgs_frame_info": _lib.FrameInfo, "fhtgs_intermediates": _lib.Intermediates,
               "fhtgs_tuning": _lib.Tuning, "fhtgs_server_config": _lib.ServerConfig, "fhtgs_eye": _lib.Eye,
               "fhtgs_request": _lib.Request, "fhtgs_completion": _lib.Completion,
               "fhtgs_server_stats": _lib.ServerStats, "fhtgs_group_completion": _lib.GroupCompletion}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        ctype = "struct fhtgs_tuning" if cname == "fhtgs_tuning" else cname
        lines.append(f'printf("{cname} size %zu\\n", sizeof({ctype}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({ctype}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, f"{cname}.{fname}"


def test_server_entry_points_fail_cleanly_without_a_device():
    lib = _lib.load()
    cfg = _lib.ServerConfig(0, 2, 8, 0, 0)
    out = _lib.vp()
    st = lib.fhtgs_server_create(C.byref(cfg), C.byref(out))
    if st == 0:  # a GPU is present: nothing to check here
        lib.fhtgs_server_destroy(out)
        pytest.skip("CUDA device present")
    assert st in (1, 2) and not out.value
    assert lib.fhtgs_server_destroy(None) == 0
    n = C.c_int32(0)
    assert lib.fhtgs_server_poll(None, None, 1, 0, C.byref(n)) == 1
    assert lib.fhtgs_server_submit(None, None, None) == 1
    bad = _lib.ServerConfig(0, 9, 8, 0, 0)
    assert lib.fhtgs_server_create(C.byref(bad), C.byref(out)) == 1
    assert b"max_in_flight" in lib.fhtgs_last_error()


def test_noalloc_sort_rejects_overlapping_buffers_before_any_device_work():
    """Partial overlaps between the no-allocation sort's buffers are refused on the host (the
    addresses below are never dereferenced); only exact in-place calls are allowed."""
    lib = _lib.load()
    n = 1000
    base = 1 << 40
    k_in, v_in = base, base + (1 << 20)
    for k_out, v_out in ((k_in + 2, base + (2 << 20)),        # keys_out shifted into keys_in
                         (base + (3 << 20), v_in + 4),        # values_out shifted into values_in
                         (v_in, base + (3 << 20)),            # keys_out on top of values_in
                         (base + (3 << 20), base + (3 << 20) + 8)):  # the two outputs overlap
        assert lib.fhtgs_sort_instances_noalloc(k_in, v_in, k_out, v_out, n, 2, 13, None) == 1
        assert b"overlap" in lib.fhtgs_last_error()


def test_server_group_entry_points_fail_cleanly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present (this checks the failure path without one)")
    lib = _lib.load()
    cfg = _lib.ServerConfig(0, 2, 8, 0, 0)
    out = _lib.vp()
    devs = (C.c_int32 * 2)(0, 0)
    assert lib.fhtgs_server_group_create(devs, 0, C.byref(cfg), C.byref(out)) == 1
    assert lib.fhtgs_server_group_create(devs, 2, C.byref(cfg), C.byref(out)) != 0  # no CUDA device here
    assert not out.value
    assert lib.fhtgs_server_group_size(None) == 0
    assert lib.fhtgs_server_group_destroy(None) == 0
    assert lib.fhtgs_server_group_submit(None, None, None, None) == 1
