# SPDX-License-Identifier: GPL-3.0-or-later
"""The batched form: domains of uneven sizes in one handle, every launch covering all members. In the FP64
form each member's result is bit-identical to the same domain run alone, and to the oracle."""
import numpy as np
import pytest

import _oracle
from cppwrf_b200 import Batch, Domain, capi
from cases import lam_case

pytestmark = pytest.mark.gpu

SIZES = [(24, 20, 14, 3), (31, 17, 14, 4), (18, 26, 14, 5), (40, 33, 14, 6)]


def test_batch_members_equal_alone_and_oracle():
    cases = [lam_case(nx=nx, ny=ny, nz=nz, seed=s) for nx, ny, nz, s in SIZES]
    b = Batch([c.g for c in cases], [c.o for c in cases])
    for m, c in enumerate(cases):
        b.upload_case(m, c)
    b.step(3)
    b.sync()
    for m, c in enumerate(cases):
        alone = Domain(c.g, c.o).upload_case(c)
        alone.step(3)
        orc = _oracle.Oracle(c)
        orc.step(3)
        for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL", "WW_M"):
            a = b.field(m, name)
            assert np.array_equal(a, alone.field(name)), (m, name)
            assert np.array_equal(a.view(np.uint64), orc.array(name).view(np.uint64)), (m, name)
        for n in range(c.o.n_scalars):
            assert np.array_equal(b.field(m, "Q_2", n).view(np.uint64), orc.array("Q_2", n).view(np.uint64)), (m, n)


def test_batch_mixed_nz_and_ideal():
    """Members with different level counts and boundary kinds in one launch sequence."""
    import cases as cs
    c1 = lam_case(nx=22, ny=18, nz=12, seed=8)
    c2 = lam_case(nx=26, ny=21, nz=17, seed=9)
    b = Batch([c1.g, c2.g], [c1.o, c2.o])
    b.upload_case(0, c1).upload_case(1, c2)
    b.step(2)
    for m, c in enumerate((c1, c2)):
        orc = _oracle.Oracle(c)
        orc.step(2)
        for name in ("U_2", "W_2", "T_2", "MU_2", "P"):
            assert np.array_equal(b.field(m, name).view(np.uint64), orc.array(name).view(np.uint64)), (m, name)


def test_batch_of_fourteen_members():
    """Fourteen members of uneven sizes and species counts in one launch per kernel (the members' descriptors in
    device memory): every member matches the oracle bit for bit."""
    cases = [lam_case(nx=14 + (m % 5), ny=12 + (m % 3), nz=10, seed=20 + m, n_moist=2 + (m % 2),
                      n_scalars=2 + (m % 2) + (m % 3)) for m in range(14)]
    b = Batch([c.g for c in cases], [c.o for c in cases])
    for m, c in enumerate(cases):
        b.upload_case(m, c)
    b.step(2)
    b.sync()
    for m, c in enumerate(cases):
        orc = _oracle.Oracle(c)
        orc.step(2)
        for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P"):
            assert np.array_equal(b.field(m, name).view(np.uint64), orc.array(name).view(np.uint64)), (m, name)
        for n in range(c.o.n_scalars):
            assert np.array_equal(b.field(m, "Q_2", n).view(np.uint64), orc.array("Q_2", n).view(np.uint64)), (m, n)


def test_batch_members_with_different_options():
    """Members whose options differ in one launch sequence (the pack runs the open-boundary variant of k_tend for
    all; each member keeps its own boundaries, Coriolis, map factors, eddy viscosities and damping): each equals the
    oracle bit for bit."""
    import cases as cs
    c1 = lam_case(nx=22, ny=18, nz=14, seed=41)
    c2 = cs.with_coriolis(lam_case(nx=26, ny=20, nz=14, seed=42, bc=(capi.OPEN, capi.OPEN)))
    c3 = cs.every_option_case()
    c4 = lam_case(nx=20, ny=24, nz=14, seed=43, diff=True, bc=(capi.OPEN, capi.PERIODIC))
    c4.o.damp_opt, c4.o.zdamp, c4.o.dampcoef = 3, 8000.0, 0.2
    members = [c1, c2, c3, c4]
    b = Batch([c.g for c in members], [c.o for c in members])
    for m, c in enumerate(members):
        b.upload_case(m, c)
    b.step(3)
    b.sync()
    for m, c in enumerate(members):
        orc = _oracle.Oracle(c, pow_mode=_oracle.POW_OWN)
        orc.step(3)
        for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL", "WW_M"):
            assert np.array_equal(b.field(m, name).view(np.uint64), orc.array(name).view(np.uint64)), (m, name)
        for n in range(c.o.n_scalars):
            assert np.array_equal(b.field(m, "Q_2", n).view(np.uint64), orc.array("Q_2", n).view(np.uint64)), (m, n)
