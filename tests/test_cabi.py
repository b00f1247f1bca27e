# SPDX-License-Identifier: GPL-3.0-or-later
"""The C ABI library loads without a GPU, exports every entry point of include/*.h, and its host-only
parts (layouts, cases) behave like the reference's."""
import ctypes as C
import os
import re

import numpy as np

from cppwrf_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names.update(re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(cw_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(capi.LIB_PATH)
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_layout_matches_reference_formula():
    """Layout::make (src/core/halo.cpp:12-48): pitch rounded to 32, element (0,0,0) at 8 + hy*pitch."""
    lib = capi.load()
    g = capi.grid(119, 89, 44, 15000.0, 90.0, 20000.0)
    o = capi.default_options(lib)
    L = capi.Layout()
    assert lib.cw_layout_of(C.byref(g), C.byref(o), capi.F["U_2"], C.byref(L)) == 0
    pitch = (8 + 120 + 3 + 31) // 32 * 32
    assert (L.nx, L.ny, L.nz, L.sj, L.sk) == (120, 89, 44, pitch, pitch * 95)
    assert L.offset == 8 + 3 * pitch and L.total == pitch * 95 * 44
    assert lib.cw_layout_of(C.byref(g), C.byref(o), capi.F["PB"], C.byref(L)) == 0
    assert L.uniform == 1 and L.total == 44 and L.sk == 1


def test_case_generator_is_deterministic():
    import cases
    cfg = cases.SMALL["straka_small"]
    a, La = cases.ideal_case(cfg).field("T_2")
    b, Lb = cases.ideal_case(cfg).field("T_2")
    assert np.array_equal(a, b)
    assert capi.interior(a, La).min() < -10.0  # the cold bubble


def test_create_without_gpu_reports_error():
    """cw_create on a machine without a CUDA device fails with a message instead of crashing."""
    lib = capi.load()
    g = capi.grid(16, 1, 8, 100.0, 1.0, 800.0)
    o = capi.default_options(lib)
    h = C.c_void_p()
    rc = lib.cw_create(C.byref(g), C.byref(o), C.byref(h))
    if rc == 0:  # a device is present
        lib.cw_destroy(h)
    else:
        assert lib.cw_last_error(None)
