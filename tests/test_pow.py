# SPDX-License-Identifier: GPL-3.0-or-later
"""Accuracy of cw_pow (the dycore's own pow): against glibc's pow and against a 60-digit decimal evaluation."""
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
