# SPDX-License-Identifier: GPL-3.0-or-later
"""cw_div_const, the division by the flux statement functions' constants 60 and 12 without a divide instruction
(cppwrf_b200/csrc/cw_pow.h), is the IEEE quotient bit for bit: on the host (tests/div_const_check.c, 3 x 10^7
operands per constant: random bit patterns over every exponent, quotients next to a rounding midpoint, exact
quotients and their neighbours) and on the GPU (cw_check_div_const: the device form against __ddiv_rn on 2^30
operands per constant)."""
import ctypes as C
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _host_check(n, seed, tmp_path):
    exe = str(tmp_path / "div_const_check")
    subprocess.run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-o", exe, os.path.join(HERE, "div_const_check.c"),
                    "-lm"], check=True)
    out = subprocess.run([exe, str(n), str(seed)], check=True, capture_output=True, text=True).stdout
    last = out.strip().splitlines()[-1].split()
    return int(last[1]), int(last[3]), out


def test_div_const_equals_ieee_division_on_host(tmp_path):
    bad, checked, out = _host_check(30_000_000, 12345, tmp_path)
    assert checked == 60_000_000
    assert bad == 0, out


@pytest.mark.gpu
def test_div_const_equals_ieee_division_on_gpu():
    from cppwrf_b200 import capi
    lib = capi.load()
    bad = C.c_ulonglong()
    checked = C.c_ulonglong()
    assert lib.cw_check_div_const(C.c_ulonglong(1 << 30), C.c_ulonglong(2024), C.byref(checked), C.byref(bad)) == 0
    assert checked.value == 2 * (1 << 30)
    assert bad.value == 0
