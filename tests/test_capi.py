"""The C-ABI library: it loads without a GPU and exports every entry point
that include/*.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(inc, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(fl_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from fluidity_b200 import build, capi
    build.build()
    return capi.load()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "fl_split_sweep" in names and "fl_split_solve" in names and "fl_simulate" in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(lib, name):
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_binding_covers_header():
    from fluidity_b200 import capi
    assert set(declared_functions()) <= set(capi.PROTOTYPES), "ctypes binding misses a symbol"


def test_version_and_error_string(lib):
    assert lib.fl_version() >= 100
    assert isinstance(lib.fl_last_error_string(), bytes)


def test_argument_errors_without_gpu(lib):
    """Invalid arguments are rejected before any CUDA call."""
    from fluidity_b200 import capi
    g = capi.Grid.make((3,))
    rc = lib.fl_split_sweep(ctypes.byref(g), 0, ctypes.c_void_p(8), ctypes.c_void_p(16), 1.4,
                            0.1, 0, 0, None, None)
    assert rc == capi.FL_EINVAL
    assert b"n[0]" in lib.fl_last_error_string()
    g = capi.Grid.make((16, 16))
    rc = lib.fl_split_sweep(ctypes.byref(g), 2, ctypes.c_void_p(8), ctypes.c_void_p(16), 1.4,
                            0.1, 0, 0, None, None)
    assert rc == capi.FL_EINVAL
    rc = lib.fl_split_sweep(ctypes.byref(g), 0, ctypes.c_void_p(8), ctypes.c_void_p(16), 1.4,
                            0.1, 1 << 9, 0, None, None)
    assert rc == capi.FL_EINVAL and b"policy" in lib.fl_last_error_string()
    rc = lib.fl_split_sweep(ctypes.byref(g), 0, None, ctypes.c_void_p(16), 1.4, 0.1, 0, 0,
                            None, None)
    assert rc == capi.FL_EINVAL
    assert lib.fl_state_bytes(ctypes.byref(g), capi.FL_DTYPE_F32) == 4 * 256 * 4


def test_policy_bits():
    from fluidity_b200 import capi
    assert capi.policy_bits() == 0
    assert capi.policy_bits("f32", "force", "superbee", "basic", False) == 1 | 2 | 8 | 16 | 32
