# SPDX-License-Identifier: GPL-3.0-or-later
"""The reference's dycore check 1 on the oracle (CPU): the map-factor form is invariant -- squall2d with a constant
map factor m = 2 and dx = 2000 m equals m = 1 and dx = 1000 m bit for bit (emdiv = 0). The GPU path is pinned to
the oracle bit for bit, and tests/test_properties_gpu.py runs the same check there."""
import numpy as np

import _oracle
import cases
from cppwrf_b200 import capi


def scaled_pair():
    cfg = dict(cases.golden_config("squall2d"))
    a = cases.ideal_case(cfg, emdiv=0.0)
    b = cases.ideal_case(dict(cfg, dx=2.0 * cfg["dx"], dy=2.0 * cfg["dy"]), emdiv=0.0)
    for name in capi.FIELDS:
        if name.startswith("Q_"):
            continue
        x, _ = a.field(name)
        y, _ = b.field(name)
        y[:] = x
    for which in ("Q_1", "Q_2"):
        for n in range(a.o.n_scalars):
            x, _ = a.field(which, n)
            y, _ = b.field(which, n)
            y[:] = x
    for name in ("MSFTX", "MSFTY", "MSFUX", "MSFUY", "MSFVX", "MSFVY"):
        y, _ = b.field(name)
        y[:] = 2.0
    y, _ = b.field("MSFVX_INV")
    y[:] = 0.5
    return a, b


def test_map_factor_invariance_oracle():
    a, b = scaled_pair()
    oa, ob = _oracle.Oracle(a, pow_mode=_oracle.POW_OWN), _oracle.Oracle(b, pow_mode=_oracle.POW_OWN)
    oa.step(10)
    ob.step(10)
    for name in ["U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL", "RAINNC"]:
        assert np.array_equal(oa.array(name).view(np.uint64), ob.array(name).view(np.uint64)), name
    assert not np.array_equal(oa.array("W_2"), cases.ideal_case(dict(cases.golden_config("squall2d")),
                                                                 emdiv=0.0).field("W_2")[0])  # it moved
