# SPDX-License-Identifier: GPL-3.0-or-later
"""Failure detection and checkpoint / resume on the GPU path, without faulting the GPU: a non-finite value seeded
into the host input is found and named (CPPWRF's run.check_nonfinite_every_step); a run restarted from the
downloaded state continues bit-identically (the reference's restart test)."""
import ctypes as C

import numpy as np
import pytest

from cppwrf_b200 import Domain, capi
from cases import lam_case

pytestmark = pytest.mark.gpu


def test_nonfinite_value_is_found_and_named():
    case = lam_case(nx=30, ny=24, nz=12, seed=21)
    d = Domain(case.g, case.o).upload_case(case)
    d.step(1)
    assert d.check_finite() is None
    L = d.layout("T_2")
    t = d.field("T_2")
    t[L.offset + 5 * L.si + 4 * L.sj + 3 * L.sk] = np.nan
    d.upload("T_2", t)
    Lq = d.layout("Q_2", 2)
    q = d.field("Q_2", 2)
    q[Lq.offset + 1 * Lq.si + 1 * Lq.sj + 1 * Lq.sk] = np.inf
    d.upload("Q_2", q, 2)
    assert d.check_finite() == ("T_2", 0, 5, 4, 3)  # T_2 comes before the species in the scan order
    t[L.offset + 5 * L.si + 4 * L.sj + 3 * L.sk] = 300.0 - 300.0
    d.upload("T_2", t)
    assert d.check_finite() == ("Q_2", 2, 1, 1, 1)


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED], ids=["fp64", "mixed"])
def test_restart_from_downloaded_state_is_bit_identical(precision):
    case = lam_case(nx=33, ny=26, nz=14, seed=22, diff=True, precision=precision)
    a = Domain(case.g, case.o).upload_case(case)
    a.step(4)
    b = Domain(case.g, case.o).upload_case(case)
    b.step(2)
    saved = {name: b.field(name) for name in capi.STATE_FIELDS}
    saved_q = [b.field("Q_2", n) for n in range(case.o.n_scalars)]
    c = Domain(case.g, case.o).upload_case(case)
    for name, arr in saved.items():
        c.upload(name, arr)
    for n, arr in enumerate(saved_q):
        c.upload("Q_2", arr, n)
    assert c.lib.cw_set_lbc_time(c.h, C.c_double(2 * case.g.dt)) == 0  # the boundary clock after two steps
    c.step(2)
    for name in capi.STATE_FIELDS:
        assert np.array_equal(c.field(name).view(np.uint64), a.field(name).view(np.uint64)), name
    for n in range(case.o.n_scalars):
        assert np.array_equal(c.field("Q_2", n).view(np.uint64), a.field("Q_2", n).view(np.uint64)), n
