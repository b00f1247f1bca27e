# SPDX-License-Identifier: GPL-3.0-or-later
"""Run outputs in CPPWRF's formats, without a GPU.

- The oracle's diagnostics (dyn::Diagnostics::compute in the reference CPU build's reduction order) equal every
  row of the reference's golden diag.csv files bit for bit (steps 0, 1, 2 of the four regression cases).
- cw_diag_header / cw_diag_format_row reproduce the golden diag.csv text (io::DiagWriter's number formatting).
- cw_snapshot_write_host, given the oracle's state at the golden step, writes a snap_000002.bin whose every
  variable has the golden's SHA-256 and a snap_000002.json identical to the golden's text.
- squall2d (moist convection, Kessler microphysics after the RK3 loop): the case generator, the oracle's physics
  coupling and the writer reproduce that golden too (theta_m, qv, qc, qr, rainnc, rainncv included).
- The moist variables of a snapshot (dry theta from theta_m, theta_m, the species under their names).
"""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

import _oracle
import cases
from cppwrf_b200 import capi

CASES = ["straka", "warm_bubble", "igw", "rest_state", "squall2d"]


def _golden_rows(name):
    lines = cases.GOLDEN["cases"][name]["diag_csv"]
    return lines[0], [l.split(",") for l in lines[1:]]


@pytest.mark.parametrize("name", CASES)
def test_oracle_diagnostics_match_golden_diag_csv(name):
    cfg = cases.golden_config(name)
    orc = _oracle.Oracle(cases.ideal_case(cfg), pow_mode=_oracle.POW_GLIBC)
    _, rows = _golden_rows(name)
    done = 0
    for r in rows:
        step = int(r[0])
        orc.step(step - done)
        done = step
        got = orc.diagnostics()
        want = [float(x) for x in r[2:10]]
        bad = [(k, got[k], w) for k, w in zip(capi.DIAG_KEYS, want) if got[k] != w]
        assert not bad, f"{name} step {step}: {bad}"


@pytest.mark.parametrize("name", CASES)
def test_diag_csv_text(name):
    lib = capi.load()
    header, rows = _golden_rows(name)
    assert capi.diag_header(lib) == header
    for line, r in zip(cases.GOLDEN["cases"][name]["diag_csv"][1:], rows):
        d = dict(zip(capi.DIAG_KEYS, [float(x) for x in r[2:10]]))
        assert capi.diag_row(int(r[0]), float(r[1]), d, float(r[10]), lib) == line


def _snapshot_fields(orc):
    names = ("U_2", "V_2", "W_2", "T_2", "P", "PH_2", "MU_2", "PB", "PHB", "T_INIT", "MUB", "RAINNC", "RAINNCV")
    return {n.lower(): orc.array(n) for n in names}


def _read_snapshot(directory, step):
    base = os.path.join(directory, "snap_%06d" % step)
    text = open(base + ".json").read()
    meta = json.loads(text)
    raw = open(base + ".bin", "rb").read()
    out = {}
    for v in meta["variables"]:
        out[v["name"]] = np.frombuffer(raw[v["offset"]:v["offset"] + v["nbytes"]], dtype="<f8").reshape(v["shape"])
    return text, meta, out


@pytest.mark.parametrize("name", CASES)
def test_snapshot_writer_matches_golden(name, tmp_path):
    gold = cases.GOLDEN["cases"][name]
    cfg = gold["config"]
    case = cases.ideal_case(cfg)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(gold["step"])
    qs = [orc.array("Q_2", n) for n in range(case.o.n_scalars)]
    capi.snapshot_write_host(tmp_path, gold["step"], float(gold["time"]), case.g, case.o, _snapshot_fields(orc), qs)
    text, meta, vars_ = _read_snapshot(str(tmp_path), gold["step"])
    assert text == gold["snap_json"]
    for var, ref in gold["variables"].items():
        assert hashlib.sha256(vars_[var].astype("<f8").tobytes()).hexdigest() == ref["sha256"], var
    assert sorted(os.listdir(tmp_path)) == ["snap_000002.bin", "snap_000002.json"]  # no temporaries left


def test_snapshot_moist_variables(tmp_path):
    """theta = theta_m / (1 + rvovrd qv) (dry), theta_m, and each species under its name after the dry ones."""
    case = cases.lam_case(seed=5, nx=16, ny=12, nz=10)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(1)
    ns = case.o.n_scalars
    names = ["qv"] + [f"tr{n}" for n in range(1, ns)]
    qs = [orc.array("Q_2", n) for n in range(ns)]
    capi.snapshot_write_host(tmp_path, 7, 90.0, case.g, case.o, _snapshot_fields(orc), qs, names)
    text, meta, v = _read_snapshot(str(tmp_path), 7)
    assert [x["name"] for x in meta["variables"]] == ["u", "v", "w", "th_pert", "theta", "theta_m", "p", "p_pert",
                                                       "ph", "mu", "mu_pert", "z_m"] + names
    assert meta["step"] == 7 and meta["time"] == 90.0
    t = capi.interior(orc.array("T_2"), orc.layout("T_2"))
    qv = capi.interior(qs[0], orc.layout("Q_2", 0))
    rvovrd = 461.6 / 287.0
    theta = (t + 300.0) / (1.0 + rvovrd * qv)
    assert np.array_equal(v["theta"], theta)
    assert np.array_equal(v["theta_m"], t + 300.0)
    for n in range(ns):
        assert np.array_equal(v[names[n]], capi.interior(qs[n], orc.layout("Q_2", n)))
    # default names: qv, then q<n>
    capi.snapshot_write_host(tmp_path, 8, 91.0, case.g, case.o, _snapshot_fields(orc), qs)
    _, meta, _ = _read_snapshot(str(tmp_path), 8)
    assert [x["name"] for x in meta["variables"]][12:] == ["qv"] + [f"q{n}" for n in range(1, ns)]


def test_snapshot_refuses_missing_arrays(tmp_path):
    lib = capi.load()
    cfg = dict(cases.golden_config("rest_state"), nx=8, ny=8, nz=6)
    case = cases.ideal_case(cfg)
    f = capi.SnapshotFields()
    rc = lib.cw_snapshot_write_host(str(tmp_path).encode(), 0, 0.0, C.byref(case.g), C.byref(case.o), C.byref(f), None)
    assert rc != 0 and b"missing" in lib.cw_output_last_error()
