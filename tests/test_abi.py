"""The C-ABI library: it loads and exports every entry point include/sqb200.h declares, and
fails cleanly (status code, no crash, no CPU fallback) where no CUDA device exists."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden, golden_basis, gpu_available, load_sqb200

HEADER = os.path.join(ROOT, "include", "sqb200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char \*|double)\s*\*?\s*(sqb200_\w+)\s*\(", txt, re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "sqb200_jk_create" in names and "sqb200_jk_build" in names
    assert len(names) >= 8


def test_library_exports_every_declared_symbol():
    sqb = load_sqb200()
    L = sqb.load_library()
    for name in declared():
        assert hasattr(L, name), name


def test_python_binding_covers_exports():
    sqb = load_sqb200()
    assert set(declared()) <= set(sqb.engine.EXPORTS) | {"sqb200_jk_build_noalloc"}


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly():
    sqb = load_sqb200()
    g = golden("water_321g")
    with pytest.raises(sqb.SQB200Error) as e:
        sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])
    assert "error -5" in str(e.value) or "error -4" in str(e.value)


def test_invalid_arguments_rejected():
    sqb = load_sqb200()
    L = sqb.load_library()
    ctx = ctypes.c_void_p()
    z = np.zeros(3, np.int32)
    f = np.zeros(3)
    rc = L.sqb200_jk_create(ctypes.byref(ctx), 0, z, z, f, f, f, None, 0)
    assert rc == -1
    assert b"nbf" in L.sqb200_last_error()
