"""The C-ABI library loads and exports every entry point include/stir_b200.h declares (no GPU calls)."""
import ctypes
import os
import re

import pytest

from stir_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "stir_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(b200rt_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "b200rt_create" in syms and "b200rt_forward_project_dev" in syms and len(syms) >= 14


def test_library_exports_every_declared_symbol():
    lib = _abi.load_library()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    bound = {name for name, _, _ in _abi.EXPORTS}
    assert set(declared_symbols()) <= bound, set(declared_symbols()) - bound


def test_struct_layout_matches_header():
    # b200rt_geometry: 10 scalars, 6 ints, 3 arrays of 255, 6 ints, 6 floats, 7 ints, the TOF cut-off
    assert ctypes.sizeof(_abi.Geometry) == 4 * (10 + 6 + 3 * 255 + 6 + 6 + 7 + 1)
    assert ctypes.sizeof(_abi.Info) == 5 * 8 + 4 * 4
    assert ctypes.sizeof(_abi.Prior) == 6 * 4 + 8


def test_null_arguments_are_rejected_without_touching_the_gpu():
    lib = _abi.load_library()
    assert lib.b200rt_create(None, 0, None) == _abi.ERR_INVALID_ARGUMENT
    out = ctypes.c_void_p()
    assert lib.b200rt_create(None, 0, ctypes.byref(out)) == _abi.ERR_INVALID_ARGUMENT
    assert lib.b200rt_last_error(None).decode() == "null geometry"
    assert lib.b200rt_forward_project_dev(None, None, None, 0, 1, None) == _abi.ERR_INVALID_ARGUMENT
    assert lib.b200rt_get_info(None, None) == _abi.ERR_INVALID_ARGUMENT
    lib.b200rt_destroy(None)


def test_python_constants_match_header():
    """Every B200RT_* constant the header defines that the Python binding mirrors (same name without the prefix)
    has the same value there."""
    src = open(os.path.join(ROOT, "include", "stir_b200.h")).read()
    defines = dict(re.findall(r"^#define B200RT_([A-Z0-9_]+)\s+\(?(-?\d+)u?\)?", src, flags=re.M))
    checked = 0
    for name, value in defines.items():
        if hasattr(_abi, name):
            assert getattr(_abi, name) == int(value), name
            checked += 1
    assert checked >= 20
