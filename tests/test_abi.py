"""CPU tests of the C-ABI boundary: the library loads, exports every symbol include/*.h declares,
and rejects invalid grids on the host before touching a device."""
import ctypes
import os
import re

import pytest

from ds2d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(ds2d_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_loads_and_exports_header():
    lib = _lib.load()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert declared == set(_lib.EXPORTS) | (declared - set(_lib.EXPORTS))
    for name in _lib.EXPORTS:
        assert name in declared


@pytest.mark.parametrize("bad", [
    dict(allnx=0), dict(nx=500), dict(pml=4), dict(dt=0.0), dict(nt=0),
])
def test_create_rejects_bad_grid(bad):
    lib = _lib.load()
    g = dict(allnx=100, allnz=50, nx=80, pml=10, nt=10, dx=10.0, dz=10.0, dt=0.001)
    g.update(bad)
    grid = _lib.Grid(g["allnx"], g["allnz"], g["nx"], g["pml"], g["nt"], g["dx"], g["dz"], g["dt"])
    opts = _lib.Opts(0, 0, 1, 10, 0, 0)
    h = ctypes.c_void_p()
    rc = lib.ds2d_create(ctypes.byref(grid), ctypes.byref(opts), ctypes.byref(h))
    assert rc == _lib.DS2D_E_ARG
    assert not h.value
    assert lib.ds2d_last_error(None)


def test_null_context_calls_fail_cleanly():
    lib = _lib.load()
    assert lib.ds2d_set_models(None, None, None, None) == _lib.DS2D_E_ARG
    assert lib.ds2d_destroy(None) == _lib.DS2D_OK
    assert lib.ds2d_last_cell_updates(None) == 0.0
