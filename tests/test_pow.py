# SPDX-License-Identifier: GPL-3.0-or-later
"""Accuracy of the dycore's own pow, exp, log, sin and cos (cw_pow.h): against glibc's and against 60-digit decimal evaluations."""
import ctypes as C
import math
import os
import subprocess
from decimal import Decimal, getcontext

import numpy as np

import _oracle

ROOT = _oracle.ROOT
SRC = r"""
#include "cw_pow.h"
double cwp(double x, double y) { return cw_pow(x, y); }
double cwe(double x) { return cw_exp(x); }
double cws(double x) { return cw_sin(x); }
double cwl(double x) { return cw_log(x); }
double cwc(double x) { return cw_cos(x); }
"""


def _lib(tmp_path):
    src = tmp_path / "p.c"
    src.write_text(SRC)
    so = tmp_path / "libp.so"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I",
                    os.path.join(ROOT, "cppwrf_b200", "csrc"), str(src), "-o", str(so), "-lm"], check=True)
    lib = C.CDLL(str(so))
    lib.cwp.restype = C.c_double
    lib.cwp.argtypes = [C.c_double, C.c_double]
    for f in (lib.cwe, lib.cws, lib.cwl, lib.cwc):
        f.restype = C.c_double
        f.argtypes = [C.c_double]
    return lib


def _ulp_err(x, y, got):
    getcontext().prec = 60
    exact = Decimal(x) ** Decimal(y) if x > 0 else None
    ref = float(exact)
    u = math.ulp(ref)
    return abs(Decimal(got) - exact) / Decimal(u)


def test_pow_within_half_ulp_plus(tmp_path):
    lib = _lib(tmp_path)
    rng = np.random.default_rng(1)
    y = 1004.5 / 717.5
    worst = 0
    for x in rng.uniform(0.05, 1.3, 400):
        e = _ulp_err(float(x), y, lib.cwp(float(x), y))
        worst = max(worst, e)
    assert worst < Decimal("0.5001"), worst


def test_pow_agrees_with_glibc_to_one_ulp(tmp_path):
    lib = _lib(tmp_path)
    rng = np.random.default_rng(2)
    for x, y in zip(rng.uniform(1e-3, 50, 2000), rng.uniform(-4, 4, 2000)):
        a, b = lib.cwp(x, y), math.pow(x, y)
        assert abs(a - b) <= math.ulp(b), (x, y, a, b)


def test_pow_special_values(tmp_path):
    lib = _lib(tmp_path)
    assert lib.cwp(2.0, 0.0) == 1.0
    assert lib.cwp(1.0, 7.3) == 1.0
    assert lib.cwp(0.0, 1.4) == 0.0
    assert math.isinf(lib.cwp(0.0, -1.4))
    assert math.isnan(lib.cwp(-2.0, 1.4))
    assert lib.cwp(-2.0, 3.0) == -8.0
    assert math.isinf(lib.cwp(math.inf, 1.4))
    assert lib.cwp(1e-310, 1.4) == math.pow(1e-310, 1.4)


def _dec_sin(x):
    getcontext().prec = 60
    x = Decimal(x)
    s, term, n = Decimal(0), x, 1
    while term != 0 and (s == 0 or abs(term) > abs(s) * Decimal(10) ** -58):
        s += term
        term = -term * x * x / ((n + 1) * (n + 2))
        n += 2
    return s


def test_sin_within_half_ulp_plus(tmp_path):
    """cw_sin on damp_opt 3's range [0, pi/2] (and to |x| <= 2): within 0.5001 ulp of the exact value."""
    lib = _lib(tmp_path)
    rng = np.random.default_rng(3)
    worst = Decimal(0)
    for x in list(rng.uniform(0.0, 2.0, 400)) + [1e-300, 1e-8, math.pi / 2]:
        got = lib.cws(float(x))
        exact = _dec_sin(float(x))
        worst = max(worst, abs(Decimal(got) - exact) / Decimal(math.ulp(float(exact))))
    assert worst < Decimal("0.5001"), worst
    assert math.copysign(1.0, lib.cws(-0.0)) == -1.0 and lib.cws(-1.0) == -lib.cws(1.0)
    assert math.isnan(lib.cws(2.5)) and math.isnan(lib.cws(math.nan))


def test_sin_agrees_with_glibc_to_one_ulp(tmp_path):
    lib = _lib(tmp_path)
    for x in np.random.default_rng(4).uniform(0.0, math.pi / 2, 5000):
        a, b = lib.cws(float(x)), math.sin(float(x))
        assert abs(a - b) <= math.ulp(b), (x, a, b)


def test_exp_within_half_ulp_plus(tmp_path):
    """cw_exp (the Kessler saturation vapour pressure) within 0.5001 ulp of the exact value."""
    lib = _lib(tmp_path)
    getcontext().prec = 60
    worst = Decimal(0)
    for x in np.random.default_rng(5).uniform(-30.0, 30.0, 400):
        exact = Decimal(float(x)).exp()
        worst = max(worst, abs(Decimal(lib.cwe(float(x))) - exact) / Decimal(math.ulp(float(exact))))
    assert worst < Decimal("0.5001"), worst
    assert lib.cwe(0.0) == 1.0 and math.isinf(lib.cwe(800.0)) and lib.cwe(-800.0) == 0.0 and math.isnan(lib.cwe(math.nan))


def test_log_within_half_ulp_plus(tmp_path):
    """cw_log (hypsometric_opt 2: log of the ratio of the pressures at a layer's faces, just above 1, and any
    positive argument) within 0.5001 ulp of the exact value."""
    lib = _lib(tmp_path)
    getcontext().prec = 60
    rng = np.random.default_rng(6)
    xs = list(rng.uniform(1.0, 1.5, 300)) + list(np.exp(rng.uniform(-700.0, 700.0, 200))) + [1e-310, 0.5, 2.0, 1 + 2**-52]
    worst = Decimal(0)
    for x in xs:
        exact = Decimal(float(x)).ln()
        worst = max(worst, abs(Decimal(lib.cwl(float(x))) - exact) / Decimal(math.ulp(float(exact))))
    assert worst < Decimal("0.5001"), worst
    assert lib.cwl(1.0) == 0.0 and math.isinf(lib.cwl(0.0)) and lib.cwl(0.0) < 0
    assert math.isnan(lib.cwl(-1.0)) and math.isnan(lib.cwl(math.nan)) and lib.cwl(math.inf) == math.inf


def test_log_agrees_with_glibc_to_one_ulp(tmp_path):
    lib = _lib(tmp_path)
    for x in np.random.default_rng(7).uniform(1.0, 1.5, 5000):
        a, b = lib.cwl(float(x)), math.log(float(x))
        assert abs(a - b) <= math.ulp(b), (x, a, b)


def _dec_cos(x):
    getcontext().prec = 60
    x = Decimal(x)
    s, term, n = Decimal(0), Decimal(1), 0
    while term != 0 and (s == 0 or abs(term) > abs(s) * Decimal(10) ** -58):
        s += term
        term = -term * x * x / ((n + 1) * (n + 2))
        n += 2
    return s


def test_cos_within_half_ulp_plus(tmp_path):
    """cw_cos on damp_opt 1's range [0, pi/2] (and to |x| <= 2), near pi/2 too: within 0.5001 ulp of the exact value."""
    lib = _lib(tmp_path)
    rng = np.random.default_rng(8)
    xs = list(rng.uniform(0.0, 2.0, 400)) + list(math.pi / 2 - rng.uniform(0.0, 1e-3, 100)) + \
        [0.0, 1e-8, math.pi / 4, math.nextafter(math.pi / 4, 1.0), math.pi / 2, math.nextafter(math.pi / 2, 2.0)]
    worst = Decimal(0)
    for x in xs:
        got = lib.cwc(float(x))
        exact = _dec_cos(float(x))
        worst = max(worst, abs(Decimal(got) - exact) / Decimal(math.ulp(float(exact))))
    assert worst < Decimal("0.5001"), worst
    assert lib.cwc(-1.0) == lib.cwc(1.0) and lib.cwc(0.0) == 1.0
    assert math.isnan(lib.cwc(2.5)) and math.isnan(lib.cwc(math.nan))


def test_cos_agrees_with_glibc_to_one_ulp(tmp_path):
    lib = _lib(tmp_path)
    for x in np.random.default_rng(9).uniform(0.0, math.pi / 2, 5000):
        a, b = lib.cwc(float(x)), math.cos(float(x))
        assert abs(a - b) <= math.ulp(b), (x, a, b)
