# SPDX-License-Identifier: GPL-3.0-or-later
"""Run outputs of the device state in CPPWRF's formats.

- cw_diagnostics of an FP64 handle equals the oracle's diagnostics (the reference CPU build's reduction order,
  cw_pow in both) bit for bit, every step; at step 0 it equals the reference's golden diag.csv row, to the bit
  except total_energy (glibc's pow there: relative 1e-14).
- cw_snapshot_write of the device state after the golden run writes the golden's JSON text and the same
  binary file as the host writer given the oracle's state.
- Moist (theta_m, all species), batched and mixed-precision handles.
"""
import os

import numpy as np
import pytest

import _oracle
import cases
from cases import lam_case
from cppwrf_b200 import Batch, Domain, capi

pytestmark = pytest.mark.gpu
CASES = ["straka", "warm_bubble", "igw", "rest_state", "squall2d"]


def _same(a, b):
    return all(np.float64(a[k]).view(np.uint64) == np.float64(b[k]).view(np.uint64) for k in capi.DIAG_KEYS)


@pytest.mark.parametrize("name", CASES)
def test_diagnostics_bit_exact_with_oracle_and_golden(name):
    gold = cases.GOLDEN["cases"][name]
    case = cases.ideal_case(gold["config"])
    dom = Domain(case.g, case.o).upload_case(case)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    rows = [l.split(",") for l in gold["diag_csv"][1:]]
    for r in rows:
        step = int(r[0])
        if step > 0:
            dom.step(1)
            orc.step(1)
        got, want = dom.diagnostics(), orc.diagnostics()
        assert _same(got, want), f"{name} step {step}: gpu {got} oracle {want}"
        if step == 0:
            ref = dict(zip(capi.DIAG_KEYS, [float(x) for x in r[2:10]]))
            for k in capi.DIAG_KEYS[:7]:
                assert got[k] == ref[k], (k, got[k], ref[k])
            assert abs(got["total_energy"] - ref["total_energy"]) <= 1e-14 * abs(ref["total_energy"])


@pytest.mark.parametrize("name", CASES)
def test_snapshot_of_device_state(name, tmp_path):
    gold = cases.GOLDEN["cases"][name]
    case = cases.ideal_case(gold["config"])
    dom = Domain(case.g, case.o).upload_case(case)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    dom.step(gold["step"])
    orc.step(gold["step"])
    dev, host = tmp_path / "dev", tmp_path / "host"
    dom.snapshot(dev, gold["step"], float(gold["time"]))
    names = ("U_2", "V_2", "W_2", "T_2", "P", "PH_2", "MU_2", "PB", "PHB", "T_INIT", "MUB", "RAINNC", "RAINNCV")
    fields = {n.lower(): orc.array(n) for n in names}
    qs = [orc.array("Q_2", n) for n in range(case.o.n_scalars)]
    capi.snapshot_write_host(host, gold["step"], float(gold["time"]), case.g, case.o, fields, qs)
    assert open(dev / "snap_000002.json").read() == gold["snap_json"]
    assert open(dev / "snap_000002.bin", "rb").read() == open(host / "snap_000002.bin", "rb").read()


def test_diagnostics_moist_and_batched():
    c1 = lam_case(nx=26, ny=21, nz=14, seed=51, diff=True)
    c2 = lam_case(nx=19, ny=23, nz=11, seed=52, n_moist=2, n_scalars=4)
    b = Batch([c1.g, c2.g], [c1.o, c2.o])
    b.upload_case(0, c1).upload_case(1, c2)
    orcs = [_oracle.Oracle(c, pow_mode=_oracle.POW_OWN) for c in (c1, c2)]
    for _ in range(3):
        b.step(1)
        for m, orc in enumerate(orcs):
            orc.step(1)
            got, want = b.diagnostics(m), orc.diagnostics()
            assert _same(got, want), f"member {m}: gpu {got} oracle {want}"
            assert got["max_abs_q"] > 0


def test_diagnostics_mixed_close_to_fp64_and_nonfinite():
    c64 = lam_case(nx=40, ny=32, nz=20, seed=53)
    c32 = lam_case(nx=40, ny=32, nz=20, seed=53, precision=capi.MIXED)
    a = Domain(c64.g, c64.o).upload_case(c64)
    m = Domain(c32.g, c32.o).upload_case(c32)
    a.step(5)
    m.step(5)
    da, dm = a.diagnostics(), m.diagnostics()
    for k in ("dry_mass", "theta_mass", "total_energy"):
        assert abs(da[k] - dm[k]) <= 1e-6 * abs(da[k]), k
    for k in ("max_abs_u", "max_abs_v", "max_abs_w", "max_abs_q"):
        assert abs(da[k] - dm[k]) <= 1e-3 * abs(da[k]), k
    # a non-finite value makes its field's maximum +Inf (absnan)
    u = a.field("U_2")
    L = a.layout("U_2")
    u[L.offset + 5 + 7 * L.sj + 3 * L.sk] = np.nan
    a.upload("U_2", u)
    d = a.diagnostics()
    assert d["max_abs_u"] == np.inf and np.isfinite(d["max_abs_w"])


def test_diag_csv_of_a_device_run(tmp_path):
    """A diag.csv written from device diagnostics reads like the reference's (header, one row per step)."""
    cfg = cases.SMALL["straka_small"]
    case = cases.ideal_case(cfg)
    dom = Domain(case.g, case.o).upload_case(case)
    lines = [capi.diag_header()]
    for n in range(3):
        if n:
            dom.step(1)
        lines.append(capi.diag_row(n, n * cfg["dt"], dom.diagnostics(), 0.0))
    path = os.path.join(tmp_path, "diag.csv")
    open(path, "w").write("\n".join(lines) + "\n")
    rows = [l.split(",") for l in open(path).read().splitlines()]
    assert rows[0][0] == "step" and len(rows) == 4 and all(len(r) == 11 for r in rows)
    assert [float(r[0]) for r in rows[1:]] == [0.0, 1.0, 2.0]
