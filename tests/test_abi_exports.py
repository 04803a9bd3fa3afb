"""The C-ABI library loads and exports every symbol include/chapsim_gpu.h
declares (no device calls)."""
import ctypes
import os
import re

from chapsim import gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "chapsim_gpu.h")).read()
    return sorted(set(re.findall(r"\b(chapsim_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_binding_list():
    assert _declared() == sorted(gpu.EXPORTED)


def test_library_exports_every_symbol():
    lib = ctypes.CDLL(gpu.LIB_PATH)
    for name in _declared():
        assert hasattr(lib, name), name


def test_init_rejects_bad_grid_without_gpu_work():
    lib = gpu.load_library()
    g = gpu.Grid(30, 32, 32, 1, 1)
    h = ctypes.c_void_p()
    rc = lib.chapsim_gpu_init(ctypes.byref(g), None, None, ctypes.byref(h))
    assert rc == -6 and not h.value
