# SPDX-License-Identifier: GPL-3.0-or-later
"""The mixed-precision form (FP32 bulk, FP64 column sum / tridiagonal solve / p'' relation) against the FP64
form, which is bit-identical to the oracle: relative L2 of every prognostic after a short run."""
import numpy as np
import pytest

from cppwrf_b200 import Domain, capi
import cases
from cases import lam_case

pytestmark = pytest.mark.gpu

# relative L2 bounds after 10 steps of the 3-D limited-area case (FP32 bulk arithmetic)
TOL = {"U_2": 1e-4, "V_2": 1e-3, "W_2": 1e-2, "T_2": 1e-5, "PH_2": 1e-3, "MU_2": 1e-2, "Q_2": 1e-3}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("hypso,bc", [(1, capi.SPECIFIED), (2, capi.SPECIFIED), (1, capi.OPEN)],
                         ids=["linear", "log_pressure", "open_boundaries"])
def test_mixed_close_to_fp64(hypso, bc):
    """hypsometric_opt 1 and 2 (the log-linear form's inverse density computed in double in both forms); specified
    and open lateral boundaries."""
    c64 = lam_case(nx=40, ny=32, nz=20, seed=11, bc=(bc, bc))
    c32 = lam_case(nx=40, ny=32, nz=20, seed=11, precision=capi.MIXED, bc=(bc, bc))
    c64.o.hypsometric_opt = c32.o.hypsometric_opt = hypso
    d64 = Domain(c64.g, c64.o).upload_case(c64)
    d32 = Domain(c32.g, c32.o).upload_case(c32)
    d64.step(10)
    d32.step(10)
    errs = {}
    for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2"):
        L = d64.layout(name)
        a = capi.interior(d32.field(name), L)
        b = capi.interior(d64.field(name), L)
        assert np.all(np.isfinite(a)), name
        errs[name] = rel_l2(a, b)
    L = d64.layout("Q_2", 0)
    errs["Q_2"] = rel_l2(capi.interior(d32.field("Q_2", 0), L), capi.interior(d64.field("Q_2", 0), L))
    bad = {k: v for k, v in errs.items() if not v <= TOL[k]}
    assert not bad, f"relative L2 over the bound: {bad} (all: {errs})"


def test_mixed_close_to_fp64_every_option():
    """The mixed form with the options the path accepts on at once: varying map factors with Coriolis, km_opt 4
    with damp_opt 1, the flux-limited sixth-order filter, hypsometric_opt 2."""
    def case(prec):
        c = cases.with_map_factors(lam_case(nx=40, ny=32, nz=20, seed=29, diff=True, mapped=True, precision=prec))
        c.o.km_opt, c.o.damp_opt, c.o.zdamp, c.o.dampcoef = 4, 1, 8000.0, 0.2
        c.o.diff_6th_opt, c.o.diff_6th_factor, c.o.hypsometric_opt = 2, 0.12, 2
        return c
    c64, c32 = case(capi.FP64), case(capi.MIXED)
    d64 = Domain(c64.g, c64.o).upload_case(c64)
    d32 = Domain(c32.g, c32.o).upload_case(c32)
    d64.step(10)
    d32.step(10)
    errs = {}
    for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2"):
        L = d64.layout(name)
        a = capi.interior(d32.field(name), L)
        b = capi.interior(d64.field(name), L)
        assert np.all(np.isfinite(a)), name
        errs[name] = rel_l2(a, b)
    bad = {k: v for k, v in errs.items() if not v <= TOL[k]}
    assert not bad, f"relative L2 over the bound: {bad} (all: {errs})"
