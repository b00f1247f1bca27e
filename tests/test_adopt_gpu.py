# SPDX-License-Identifier: GPL-3.0-or-later
"""cw_batch_adopt: a domain prepared in its own handle joins a running batch without a copy, and continues
exactly as it would alone (and the batch's other members are not disturbed)."""
import ctypes as C

import numpy as np
import pytest

from cppwrf_b200 import Batch, Domain, capi
from cases import lam_case

pytestmark = pytest.mark.gpu


def test_adopted_member_equals_alone():
    c1 = lam_case(nx=26, ny=21, nz=14, seed=31)
    c2 = lam_case(nx=30, ny=18, nz=14, seed=32)
    b = Batch([c1.g], [c1.o]).upload_case(0, c1)
    b.step(2)
    single = Domain(c2.g, c2.o).upload_case(c2)
    m = C.c_int()
    assert b.lib.cw_batch_adopt(b.h, single.h, C.byref(m)) == 0 and m.value == 1
    single.close()
    b.step(3)
    a1 = Domain(c1.g, c1.o).upload_case(c1)
    a1.step(5)
    a2 = Domain(c2.g, c2.o).upload_case(c2)
    a2.step(3)
    for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL"):
        assert np.array_equal(b.field(0, name).view(np.uint64), a1.field(name).view(np.uint64)), name
        assert np.array_equal(b.field(1, name).view(np.uint64), a2.field(name).view(np.uint64)), name


def test_released_member_continues_as_alone():
    """cw_batch_release: a member leaves a running batch without a copy into a handle of its own, continues there
    exactly as it would alone, and the members that stay (renumbered) are not disturbed."""
    c1 = lam_case(nx=26, ny=21, nz=14, seed=41)
    c2 = lam_case(nx=30, ny=18, nz=14, seed=42)
    c3 = lam_case(nx=20, ny=24, nz=14, seed=43)
    b = Batch([c1.g, c2.g, c3.g], [c1.o, c2.o, c3.o])
    for k, c in enumerate((c1, c2, c3)):
        b.upload_case(k, c)
    b.step(2)
    out = C.c_void_p()
    assert b.lib.cw_batch_release(b.h, 1, C.byref(out)) == 0 and out.value
    single = Domain.__new__(Domain)  # wrap the released handle
    single.lib, single.h, single.g, single.o = b.lib, out, c2.g, c2.o
    single.step(3)
    b.step(3)
    alone = {}
    for key, c in (("c1", c1), ("c2", c2), ("c3", c3)):
        alone[key] = Domain(c.g, c.o).upload_case(c)
        alone[key].step(5)
    for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL"):
        assert np.array_equal(single.field(name).view(np.uint64), alone["c2"].field(name).view(np.uint64)), name
        assert np.array_equal(b.field(0, name).view(np.uint64), alone["c1"].field(name).view(np.uint64)), name
        assert np.array_equal(b.field(1, name).view(np.uint64), alone["c3"].field(name).view(np.uint64)), name
    single.close()
