# SPDX-License-Identifier: GPL-3.0-or-later
"""Kessler microphysics after the RK3 loop (mp_physics = 1) on the GPU.

- The reference's squall-line case (Weisman-Klemp sounding, warm bubble, qv qc qr): the FP64 form equals the
  oracle (cw_pow / cw_exp in both) bit for bit, every field including the species and the surface rain, over
  enough steps for cloud and rain to form and fall.
- A limited-area case with seeded cloud and rain patches and specified boundaries (the spec zone keeps its
  columns out of the microphysics, calc_p_rho_phi then runs on the interior): bit for bit too.
- A batch of a Kessler member and a member without microphysics equals each run alone.
- The mixed form follows the FP64 form within a tolerance.
"""
import numpy as np
import pytest

import _oracle
import cases
from cases import lam_case
from cppwrf_b200 import Batch, Domain, capi
from test_parity_gpu import compare_all

pytestmark = pytest.mark.gpu


def squall(**over):
    cfg = dict(cases.golden_config("squall2d"), **over)
    return cfg, cases.ideal_case(cfg)


def test_squall2d_bit_exact_with_oracle():
    cfg, case = squall()
    dom = Domain(case.g, case.o).upload_case(case)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    for _ in range(5):  # 5 x 50 steps of 6 s: cloud after ~10 min, rain at the ground after ~20 min
        dom.step(50)
        orc.step(50)
        bad = compare_all(dom, orc, case)
        assert not bad, "\n".join(bad)
    assert orc.array("Q_2", 2).max() > 0 and orc.array("RAINNC").max() > 0


def test_lam_kessler_bit_exact_with_oracle():
    case = lam_case(nx=30, ny=24, nz=16, seed=61)
    case.o.mp_physics = 1
    dom = Domain(case.g, case.o).upload_case(case)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    dom.step(3)
    orc.step(3)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)
    rain = capi.interior(orc.array("RAINNC"), orc.layout("RAINNC"))
    assert rain.max() > 0 and np.all(rain[:, 0, :] == 0) and np.all(rain[:, :, 0] == 0)  # none in the spec zone


def test_batch_with_and_without_microphysics_equals_alone():
    c1 = lam_case(nx=26, ny=21, nz=14, seed=62)
    c1.o.mp_physics = 1
    c2 = lam_case(nx=22, ny=19, nz=14, seed=63)
    b = Batch([c1.g, c2.g], [c1.o, c2.o])
    b.upload_case(0, c1).upload_case(1, c2)
    b.step(3)
    for m, c in enumerate((c1, c2)):
        a = Domain(c.g, c.o).upload_case(c)
        a.step(3)
        for name in ("U_2", "W_2", "T_2", "P", "AL", "H_DIABATIC", "RAINNC"):
            assert np.array_equal(b.field(m, name), a.field(name)), (m, name)
        for n in range(3):
            assert np.array_equal(b.field(m, "Q_2", n), a.field("Q_2", n)), (m, n)


def test_mixed_squall2d_close_to_fp64():
    cfg, c64 = squall()
    _, c32 = squall()
    c32.o.precision = capi.MIXED
    a = Domain(c64.g, c64.o).upload_case(c64)
    m = Domain(c32.g, c32.o).upload_case(c32)
    a.step(150)
    m.step(150)
    err = {}
    for name in ("U_2", "W_2", "T_2", "PH_2"):
        x, y = a.field(name), m.field(name)
        err[name] = np.linalg.norm(x - y) / max(np.linalg.norm(x), 1e-30)
    for n, name in ((0, "qv"), (1, "qc"), (2, "qr")):
        x, y = a.field("Q_2", n), m.field("Q_2", n)
        err[name] = np.linalg.norm(x - y) / max(np.linalg.norm(x), 1e-30)
    print("mixed vs fp64 relative L2 after 15 min:", err)
    for name in ("U_2", "T_2", "PH_2", "qv"):
        assert err[name] <= 1e-3, (name, err[name])
    for name in ("W_2", "qc", "qr"):
        assert err[name] <= 1e-2, (name, err[name])
