# SPDX-License-Identifier: GPL-3.0-or-later
"""The compiled drop-in (cppwrf_b200/facade/rk3_b200.hpp, RK3B200 with dyn::RK3's signature over the C ABI) driven
by the reference's own driver objects: oracle/_ref/ref_harness_facade is the reference harness -- State,
Tendencies, BaseState, LateralBC and DiffusionDriver of the reference, built and filled as the reference's
cases::Model does -- with `dyn::RK3 rk(...)` replaced by `RK3B200 rk(...)`. After the same steps every field equals
the reference's own RK3::step (ref_harness_own, pow interposed by cw_pow) bit for bit."""
import os

import numpy as np
import pytest

import _refpath  # noqa: F401
import cases
import refdump as _refdump
from cases import lam_case
from cppwrf_b200 import capi

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(os.path.join(_refdump.REF_DIR, "ref_harness_facade")),
                                 reason="oracle/_ref/ref_harness_facade (built against the reference) not present")]


def _compare(a, b):
    assert a.keys() == b.keys()
    bad = []
    for k in a:
        if a[k].size == 0 and b[k].size == 0:
            continue
        if not np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64)):
            d = np.nonzero(a[k].view(np.uint64) != b[k].view(np.uint64))[0]
            bad.append(f"{k}: {d.size} differ, first at {d[0]}: facade {a[k][d[0]]!r} reference {b[k][d[0]]!r}")
    return bad


@pytest.mark.parametrize("kind", ["lam", "lam_diffusion", "straka"])
def test_drop_in_equals_reference_step(kind):
    if kind == "straka":
        case = cases.ideal_case(cases.SMALL["straka_small"])
    else:
        case = lam_case(seed=61, diff=kind == "lam_diffusion")
    n = 3
    facade = _refdump.run(case, n, harness="ref_harness_facade")
    ref = _refdump.run(case, n, own_pow=True)
    bad = _compare(facade, ref)
    assert not bad, "\n".join(bad)
