# SPDX-License-Identifier: GPL-3.0-or-later
"""The C ABI library loads without a GPU, exports every entry point of include/*.h, and its host-only
parts (layouts, cases) behave like the reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

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


def test_footprint_without_gpu():
    """cw_footprint needs no device: the mixed form takes about half the bytes of the FP64 form."""
    lib = capi.load()
    g = capi.grid(119, 89, 44, 15000.0, 90.0, 0.0, dy=15000.0, p_top=5000.0, bc_x=capi.SPECIFIED, bc_y=capi.SPECIFIED)
    sizes = {}
    for prec in (capi.FP64, capi.MIXED):
        o = capi.default_options(lib, flat=0, n_moist=5, n_scalars=5, lbc=1, time_step_sound=4, precision=prec)
        b = C.c_size_t()
        assert lib.cw_footprint(C.byref(g), C.byref(o), C.byref(b)) == 0
        sizes[prec] = b.value
    L = capi.Layout()
    assert lib.cw_layout_of(C.byref(g), C.byref(o), capi.F["T_2"], C.byref(L)) == 0
    assert sizes[capi.FP64] > 60 * L.total * 8  # the 3-D state, tendencies, work fields and 5 x 5 scalar arrays
    assert 0.45 < sizes[capi.MIXED] / sizes[capi.FP64] < 0.55


def test_case_clone_is_a_deep_copy():
    import cases
    c = cases.ideal_case(cases.SMALL["straka_small"])
    lib = capi.load()
    h2 = C.c_void_p()
    assert lib.cw_case_clone(c.h, C.byref(h2)) == 0
    p, L = C.POINTER(C.c_double)(), capi.Layout()
    assert lib.cw_case_field(h2, capi.F["T_2"], 0, C.byref(p), C.byref(L)) == 0
    a = np.ctypeslib.as_array(p, shape=(L.total,)).copy()
    t, _ = c.field("T_2")
    assert np.array_equal(a, t)
    t[:] = 0.0  # the clone does not share storage
    b = np.ctypeslib.as_array(p, shape=(L.total,))
    assert np.array_equal(b, a)
    g, o = capi.Grid(), capi.Options()
    assert lib.cw_case_config(h2, C.byref(g), C.byref(o)) == 0 and (g.nx, g.nz) == (c.g.nx, c.g.nz)
    lib.cw_case_destroy(h2)


def test_serve_create_without_gpu_fails_cleanly():
    lib = capi.load()
    cfg = capi.ServeConfig()
    lib.cw_serve_default_config(C.byref(cfg))
    assert cfg.hbm_budget_bytes == 150e9
    h = C.c_void_p()
    assert lib.cw_serve_create(C.byref(cfg), C.byref(h)) != 0


@pytest.mark.parametrize("change,needle", [
    (dict(damp_opt=4), "damp_opt"), (dict(hypsometric_opt=3), "hypsometric"),
    (dict(mp_physics=6), "mp_physics"),
    (dict(nz=130), "nz"), (dict(diff_opt=2), "diff_opt"), (dict(diff_opt=1, km_opt=2), "km_opt")])
def test_unsupported_options_are_refused_with_a_reason(change, needle):
    """Options outside the path are refused at cw_create with a message naming them (before any device work,
    so this runs without a GPU)."""
    lib = capi.load()
    g = capi.grid(change.get("nx", 16), 12, change.get("nz", 10), 1000.0, 5.0, 10000.0,
                  bc_x=change.get("bc_x", capi.PERIODIC), bc_y=capi.PERIODIC)
    o = capi.default_options(lib, **{k: v for k, v in change.items() if k not in ("bc_x", "nz")})
    h = C.c_void_p()
    assert lib.cw_create(C.byref(g), C.byref(o), C.byref(h)) != 0
    msg = lib.cw_last_error(None).decode()
    assert needle in msg.lower(), msg
