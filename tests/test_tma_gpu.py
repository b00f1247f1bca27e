# SPDX-License-Identifier: GPL-3.0-or-later
"""The TMA-staged scalar update and the kernels' bounded waits.

k_q_march stages each species' planes in shared memory with the tensor-memory accelerator. On 3-D domains whose rows
hold a tile's 40 staged columns (nx >= 22) the autotuner times it against the point kernel k_q_update (the first
three tuning steps run the point kernel, the next three the staged one) and keeps the faster; both give the same
bits (the tuned run equals the untuned one, which equals the oracle in the parity tests). The failure path of the
bounded waits is made on the host side with a barrier that nothing completes (no fault): the kernel gives up after
its cycle limit, the status word makes the next cw_sync fail, and the handle keeps working with unchanged results."""
import ctypes as C

import numpy as np
import pytest

from cppwrf_b200 import Domain, capi
from cases import lam_case

pytestmark = pytest.mark.gpu


def launched(dom, steps=1):
    """the kernel names of `steps` profiled steps"""
    lib = dom.lib
    nk = C.c_int()
    assert lib.cw_profile(dom.h, steps, C.byref(nk)) == 0
    names = set()
    for k in range(nk.value):
        nm, ms, n = C.create_string_buffer(64), C.c_double(), C.c_longlong()
        assert lib.cw_profile_entry(dom.h, k, nm, 64, C.byref(ms), C.byref(n)) == 0
        names.add(nm.value.decode())
    return names


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED], ids=["fp64", "mixed"])
def test_3d_domains_time_both_updates_with_the_same_bits(precision):
    case = lam_case(nx=37, ny=29, nz=16, seed=13, precision=precision)
    a = Domain(case.g, case.o).upload_case(case).set_autotune(True)
    b = Domain(case.g, case.o).upload_case(case)
    a.step(6)  # the tuning steps: the point update in shapes 0 1 2, then the staged one in shapes 2 1 0
    a.step(2)
    b.step(8)
    assert a.autotune_choice("k_q_update") in (0, 1, 2) and a.autotune_choice("k_q_march") in (0, 1, 2)
    for n in range(case.o.n_scalars):
        assert np.array_equal(a.field("Q_2", n).view(np.uint64), b.field("Q_2", n).view(np.uint64)), n
    for name in capi.STATE_FIELDS:
        assert np.array_equal(a.field(name).view(np.uint64), b.field(name).view(np.uint64)), name


def test_narrow_domains_keep_the_point_update():
    case = lam_case(nx=20, ny=16, nz=12, seed=4)  # rows of 32 elements: narrower than a tile's 40 staged columns
    d = Domain(case.g, case.o).upload_case(case).set_autotune(True)
    d.step(6)
    assert d.autotune_choice("k_q_update") in (0, 1, 2) and d.autotune_choice("k_q_march") == -1
    assert "k_q_update" in launched(d) and "k_q_march" not in launched(d)


def test_bounded_wait_gives_up_reports_and_the_handle_stays_usable():
    case = lam_case(nx=30, ny=24, nz=12, seed=8)
    a = Domain(case.g, case.o).upload_case(case)
    b = Domain(case.g, case.o).upload_case(case)
    a.step(1)
    a.sync()
    assert a.lib.cw_selftest_wait(a.h, 20_000_000) == 0  # ~10 ms of polling a barrier nothing completes
    assert a.lib.cw_sync(a.h) != 0
    assert b"timed out" in a.lib.cw_last_error(a.h)
    assert a.lib.cw_sync(a.h) == 0  # the status word was cleared
    a.step(2)
    b.step(3)
    for name in capi.STATE_FIELDS:
        assert np.array_equal(a.field(name).view(np.uint64), b.field(name).view(np.uint64)), name
    for n in range(case.o.n_scalars):
        assert np.array_equal(a.field("Q_2", n).view(np.uint64), b.field("Q_2", n).view(np.uint64)), n
