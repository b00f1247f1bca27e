# SPDX-License-Identifier: GPL-3.0-or-later
"""Test-side access to the CPU oracle (oracle/liboracle.so) and to the snapshot variables.

The oracle is the checker: only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from cppwrf_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "lib", "liboracle.so")
POW_OWN, POW_GLIBC = 0, 1
# DiagRow (src/dyn/diagnostics.hpp:13-17), in the order of the diag.csv columns, then max_abs_q
DIAG_KEYS = ("max_abs_u", "max_abs_v", "max_abs_w", "min_th_pert", "max_th_pert", "dry_mass", "theta_mass",
             "total_energy", "max_abs_q")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "lib/liboracle.so"], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        lib = C.CDLL(ORACLE_LIB)
        vp, i, dp, sz = C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_size_t
        for name, res, args in [
            ("or_create", vp, [C.POINTER(capi.Grid), C.POINTER(capi.Options)]),
            ("or_destroy", None, [vp]),
            ("or_layout", i, [vp, i, i, C.POINTER(capi.Layout)]),
            ("or_field", dp, [vp, i, i]),
            ("or_set_vertical", i, [vp, C.POINTER(capi.Vertical)]),
            ("or_set_lbc", i, [vp, i, i, dp, dp, sz]),
            ("or_set_lbc_scalar", i, [vp, i, i, dp, dp, sz]),
            ("or_set_lbc_time", i, [vp, C.c_double]),
            ("or_set_pow_mode", None, [vp, i]),
            ("or_n_sound", i, [vp]),
            ("or_step", i, [vp, i]),
            ("or_diagnostics", i, [vp, dp]),
            ("or_cfl_max", i, [vp, dp]),
        ]:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


class Oracle:
    """One domain in the oracle, filled from a capi.Case."""

    def __init__(self, case, pow_mode=POW_OWN):
        self.lib = load()
        self.g, self.o = case.g, case.o
        self.h = self.lib.or_create(C.byref(case.g), C.byref(case.o))
        if not self.h:
            raise ValueError("or_create refused the options")
        self.lib.or_set_pow_mode(self.h, pow_mode)
        v = case.vertical()
        self.lib.or_set_vertical(self.h, C.byref(v))
        for n, name in enumerate(capi.FIELDS):
            if name.startswith("Q_"):
                continue
            src, L = case.field(name)
            self.array(name)[:] = src
        for n in range(case.o.n_scalars):
            for name in ("Q_1", "Q_2", "Q_TENDF"):
                src, _ = case.field(name, n)
                self.array(name, n)[:] = src
        if case.o.lbc:
            for var in range(5):
                for side in range(4):
                    vals, tends = case.lbc(var, side)
                    self.lib.or_set_lbc(self.h, var, side, vals.ctypes.data_as(C.POINTER(C.c_double)),
                                        tends.ctypes.data_as(C.POINTER(C.c_double)), vals.size)
            for n in range(case.o.n_scalars):
                for side in range(4):
                    r = case.lbc(n, side, scalar=True)
                    if r is None:
                        continue
                    vals, tends = r
                    self.lib.or_set_lbc_scalar(self.h, n, side, vals.ctypes.data_as(C.POINTER(C.c_double)),
                                               tends.ctypes.data_as(C.POINTER(C.c_double)), vals.size)
            self.lib.or_set_lbc_time(self.h, case.lbc_time())

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.or_destroy(self.h)
            self.h = None

    def layout(self, name, n=0):
        L = capi.Layout()
        if self.lib.or_layout(self.h, capi.F[name], n, C.byref(L)) != 0:
            raise KeyError(name)
        return L

    def array(self, name, n=0):
        L = self.layout(name, n)
        return capi.as_array(self.lib.or_field(self.h, capi.F[name], n), L.total)

    def step(self, n=1):
        self.lib.or_step(self.h, n)

    def n_sound(self):
        return self.lib.or_n_sound(self.h)

    def cfl_max(self):
        """(vertical, horizontal) CFL maxima of each RK stage of the last step."""
        out = (C.c_double * 6)()
        self.lib.or_cfl_max(self.h, out)
        return [(out[2 * r], out[2 * r + 1]) for r in range(3)]

    def diagnostics(self):
        """dyn::Diagnostics::compute of the current state: a dict of the DiagRow values."""
        out = (C.c_double * 9)()
        self.lib.or_diagnostics(self.h, out)
        return dict(zip(DIAG_KEYS, list(out)))


def snapshot_vars(get, layout, g, base_get, base_layout):
    """The variables of CPPWRF's snapshot writer (src/dyn/diagnostics.cpp:110-131) for a dry state.

    get(name) -> whole-allocation array of a state field; base_get likewise for base fields.
    Returns {name: array in (k, j, i) order}.
    """
    T0, G = 300.0, 9.81
    u = capi.interior(get("U_2"), layout("U_2"))
    v = capi.interior(get("V_2"), layout("V_2"))
    w = capi.interior(get("W_2"), layout("W_2"))
    t = capi.interior(get("T_2"), layout("T_2"))
    p = capi.interior(get("P"), layout("P"))
    ph = capi.interior(get("PH_2"), layout("PH_2"))
    mu = capi.interior(get("MU_2"), layout("MU_2"))

    def base(name, L_like):
        L = base_layout(name)
        a = base_get(name)
        if L.uniform:
            vals = a[:L.nz].reshape(L.nz, 1, 1) if L.rank == 3 else a[:1].reshape(1, 1, 1)
            return np.broadcast_to(vals, L_like.shape).astype(np.float64)
        return capi.interior(a, L)

    t_init = base("T_INIT", t)
    pb = base("PB", p)
    phb = base("PHB", ph)
    mub = base("MUB", mu)
    theta = t + T0
    out = {
        "u": u, "v": v, "w": w,
        "th_pert": theta - T0 - t_init,
        "theta": theta,
        "p": p + pb,
        "p_pert": p,
        "ph": ph + phb,
        "mu": mu + mub,
        "mu_pert": mu,
        "z_m": 0.5 * (ph[:-1] + ph[1:] + phb[:-1] + phb[1:]) / G,
    }
    return out
