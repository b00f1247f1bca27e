# SPDX-License-Identifier: GPL-3.0-or-later
"""cw_download_noalloc (a download that allocates nothing; scratch in the library's device image) against
cw_download: the same bytes on two calls in a row, for FP32 (mixed) and FP64 handles, and a clear error
for an FP32 field larger than the static scratch. The file name sorts last so that it also runs after the
other GPU tests in one session; it passes alone as well."""
import ctypes as C

import numpy as np
import pytest

from cppwrf_b200 import Domain, capi
from cases import lam_case

pytestmark = pytest.mark.gpu

NAMES = [("U_2", 0), ("V_2", 0), ("W_2", 0), ("T_2", 0), ("PH_2", 0), ("MU_2", 0), ("P", 0), ("AL", 0), ("Q_2", 0),
         ("Q_2", 4)]


def _noalloc(lib, dom, name, n, out):
    return lib.cw_download_noalloc(dom.h, capi.F[name], n, out.ctypes.data_as(C.POINTER(C.c_double)), out.size)


@pytest.mark.parametrize("precision", [capi.MIXED, capi.FP64], ids=["mixed", "fp64"])
def test_noalloc_download_equals_download(precision):
    lib = capi.load()
    case = lam_case(nx=40, ny=32, nz=20, seed=7, precision=precision)
    dom = Domain(case.g, case.o).upload_case(case)
    dom.step(2)
    dom.sync()
    for name, n in NAMES:
        ref = dom.field(name, n)
        for call in range(2):
            out = np.full(ref.size, np.nan)
            assert _noalloc(lib, dom, name, n, out) == 0, (name, n, call)
            assert np.array_equal(out.view(np.uint64), ref.view(np.uint64)), (name, n, call)


def test_noalloc_rejects_fields_beyond_the_scratch():
    lib = capi.load()
    g = capi.grid(128, 128, 64, 3000.0, 18.0, 0.0, dy=3000.0, p_top=5000.0, bc_x=capi.SPECIFIED,
                  bc_y=capi.SPECIFIED)
    o = capi.default_options(lib, flat=0, n_moist=1, n_scalars=1, lbc=1, time_step_sound=6, precision=capi.MIXED)
    dom = Domain(g, o)
    L = dom.layout("T_2")
    assert L.total > capi.NOALLOC_SCRATCH_DOUBLES
    out = np.full(L.total, 7.0)
    assert _noalloc(lib, dom, "T_2", 0, out) == capi.NOALLOC_ETOOBIG
    assert np.all(out == 7.0)  # nothing copied
    small = dom.layout("MU_2")  # a 2-D field fits
    out2 = np.full(small.total, np.nan)
    assert _noalloc(lib, dom, "MU_2", 0, out2) == 0
    assert np.array_equal(out2, dom.field("MU_2"))
    bad = np.zeros(3)
    assert _noalloc(lib, dom, "MU_2", 0, bad) == capi.NOALLOC_EBADARG  # wrong count
    assert _noalloc(lib, dom, "Q_2", 5, out2) == capi.NOALLOC_EBADARG  # species out of range


def test_noalloc_rejects_another_current_device():
    """The scratch is looked up on the current device: a handle of another device is refused, not misused
    (checked only where this process sees more than one device)."""
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("one device visible: the device check has nothing to compare")
    lib = capi.load()
    case = lam_case(nx=24, ny=20, nz=12, seed=3, precision=capi.MIXED)
    lib.cw_use_device(0)
    dom = Domain(case.g, case.o).upload_case(case)
    L = dom.layout("T_2")
    out = np.full(L.total, np.nan)
    lib.cw_use_device(1)
    try:
        assert _noalloc(lib, dom, "T_2", 0, out) == capi.NOALLOC_EBADARG
    finally:
        lib.cw_use_device(0)
    assert _noalloc(lib, dom, "T_2", 0, out) == 0
