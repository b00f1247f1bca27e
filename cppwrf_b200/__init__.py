# SPDX-License-Identifier: GPL-3.0-or-later
"""B200-native WRF-ARW RK3 split-explicit dynamical core (CPPWRF's dyn::RK3 step) -- Python host mirror.

The dynamics run in libcw_dycore.so (sm_100a CUDA kernels + C++20 host runtime, include/cw_dycore.h).
This module mirrors the reference's step interface for Python callers:

    dom = Domain(grid, options)          # RK3(grid, LargeStepParams, AcousticParams, time_step_sound, ScalarParams)
    dom.upload_case(case)                # cases::Model set-up: State, BaseState, vertical arrays, boundaries
    dom.step(n)                          # RK3::step(State&, Tendencies&, const BaseState&), n times
    dom.field("U_2")                     # FieldT::download (whole allocation, CPPWRF layout)

There is no CPU path: a missing library or device raises.
"""
import ctypes as C

import numpy as np

from . import capi
from .capi import (DEFAULT, FIELDS, FP64, IGW, MIXED, PERIODIC, REST_STATE, SPECIFIED, STRAKA, SYMMETRIC,
                   WARM_BUBBLE, Case, F, Grid, Layout, Options, default_options, grid, interior)

__all__ = ["Domain", "Decomp", "Batch", "Server", "Case", "Grid", "Options", "Layout", "grid", "default_options", "interior", "capi",
           "FIELDS", "F", "PERIODIC", "SYMMETRIC", "SPECIFIED", "FP64", "MIXED", "REST_STATE", "STRAKA",
           "WARM_BUBBLE", "IGW", "DEFAULT"]


class CwError(RuntimeError):
    pass


def _check(lib, h, rc, what):
    if rc != 0:
        msg = lib.cw_last_error(h)
        raise CwError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")


class Domain:
    """One domain on the device (a handle of the C ABI)."""

    def __init__(self, g, o, lib=None):
        self.lib = lib or capi.load()
        self.g, self.o = g, o
        self.h = C.c_void_p()
        rc = self.lib.cw_create(C.byref(g), C.byref(o), C.byref(self.h))
        _check(self.lib, None, rc, "cw_create")

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.cw_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()

    def upload_case(self, case):
        _check(self.lib, self.h, self.lib.cw_upload_case(self.h, case.h), "cw_upload_case")
        return self

    def step(self, n=1):
        _check(self.lib, self.h, self.lib.cw_step(self.h, n), "cw_step")
        return self

    def sync(self):
        _check(self.lib, self.h, self.lib.cw_sync(self.h), "cw_sync")

    def n_sound(self):
        v = C.c_int()
        self.lib.cw_n_sound(self.h, C.byref(v))
        return v.value

    def launches(self):
        v = C.c_longlong()
        self.lib.cw_launch_count(self.h, C.byref(v))
        return v.value

    def layout(self, name, n=0):
        L = Layout()
        _check(self.lib, self.h, self.lib.cw_field_layout(self.h, F[name], n, C.byref(L)), "cw_field_layout")
        return L

    def field(self, name, n=0):
        L = self.layout(name, n)
        out = np.empty(L.total, dtype=np.float64)
        rc = self.lib.cw_download(self.h, F[name], n, out.ctypes.data_as(C.POINTER(C.c_double)), out.size)
        _check(self.lib, self.h, rc, "cw_download")
        return out

    def upload(self, name, arr, n=0):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        rc = self.lib.cw_upload(self.h, F[name], n, a.ctypes.data_as(C.POINTER(C.c_double)), a.size)
        _check(self.lib, self.h, rc, "cw_upload")

    def set_graph(self, on):
        self.lib.cw_set_graph(self.h, 1 if on else 0)

    def check_finite(self, member=0):
        """None when the prognostic state is finite, else (field name, species, i, j, k) of the first
        non-finite value."""
        f, n, i, j, k = (C.c_int() for _ in range(5))
        rc = self.lib.cw_check_finite(self.h, member, C.byref(f), C.byref(n), C.byref(i), C.byref(j), C.byref(k))
        _check(self.lib, self.h, 0 if rc >= 0 else rc, "cw_check_finite")
        return None if rc == 0 else (FIELDS[f.value], n.value, i.value, j.value, k.value)

    def cfl_max(self, member=0):
        """(vertical, horizontal) CFL maxima of each RK stage of the last step (cw_set_cfl_diagnostics first)."""
        v, hz = (C.c_double * 3)(), (C.c_double * 3)()
        _check(self.lib, self.h, self.lib.cw_cfl_max(self.h, member, v, hz), "cw_cfl_max")
        return list(zip(v, hz))

    def diagnostics(self, member=0):
        """dyn::Diagnostics::compute of the current state (the diag.csv values, plus max_abs_q), as a dict."""
        d = capi.Diag()
        _check(self.lib, self.h, self.lib.cw_diagnostics(self.h, member, C.byref(d)), "cw_diagnostics")
        return d.as_dict()

    def snapshot(self, directory, step, time, q_names=None, member=0):
        """Writes directory/snap_<step>.{json,bin} in CPPWRF's snapshot format."""
        na = capi.names_array(q_names)
        rc = self.lib.cw_snapshot_write(self.h, member, str(directory).encode(), step, time, na[0] if na else None)
        if rc != 0:
            raise CwError(f"cw_snapshot_write: {self.lib.cw_output_last_error().decode()}")

    def set_cfl_diagnostics(self, on=True):
        self.lib.cw_set_cfl_diagnostics(self.h, 1 if on else 0)
        return self

    def set_autotune(self, on=True):
        """The next six steps time the kernels' block shapes (two steps per shape); each kernel then keeps its
        fastest."""
        self.lib.cw_set_autotune(self.h, 1 if on else 0)
        return self

    def autotune_choice(self, kernel):
        v = C.c_int()
        self.lib.cw_autotune_choice(self.h, kernel.encode(), C.byref(v))
        return v.value


def nccl_unique_id(lib=None):
    """The 128 bytes that every rank of a decomposed domain passes to Decomp (made on one rank, sent to the others)."""
    lib = lib or capi.load()
    buf = (C.c_ubyte * 128)()
    _check(lib, None, lib.cw_nccl_unique_id(buf), "cw_nccl_unique_id")
    return bytes(buf)


def decomp_plan(g, o, px, py, rank, nranks, sets, lib=None):
    """cw_decomp_plan: the boxes crossing between `rank` and the other ranks at the fill point made of `sets`, one row
    each: role (0 packed by this rank, 1 unpacked), peer, receiving patch, owning patch, field, i0, i1, j0, j1,
    levels, offset in the send / receive region (no device)."""
    lib = lib or capi.load()
    s = (C.c_int * len(sets))(*sets)
    n = C.c_int()
    _check(lib, None, lib.cw_decomp_plan(C.byref(g), C.byref(o), px, py, rank, nranks, len(sets), s, None, 0,
                                         C.byref(n)), "cw_decomp_plan")
    out = np.zeros((max(n.value, 1), 11), dtype=np.int64)
    _check(lib, None, lib.cw_decomp_plan(C.byref(g), C.byref(o), px, py, rank, nranks, len(sets), s,
                                         out.ctypes.data_as(C.POINTER(C.c_longlong)), n.value, C.byref(n)),
           "cw_decomp_plan")
    return out[:n.value]


class Decomp:
    """One domain decomposed into px x py patches (cw_decomp_create): fields go in and out as whole-domain arrays;
    the step is RK3::step of the undecomposed domain, bit for bit. With nranks > 1 the patches are spread over
    processes (cw_decomp_create_ranked: patch t on rank t % nranks, halos over NCCL; nccl_id from nccl_unique_id on
    one rank, the same on all), or with loopback=True all held here with the ranks' exchanges through the packed
    buffers."""

    def __init__(self, g, o, px, py, lib=None, rank=0, nranks=1, nccl_id=None, loopback=False):
        self.lib = lib or capi.load()
        self.g, self.o = g, o
        self.h = C.c_void_p()
        if nranks == 1 and not loopback:
            rc = self.lib.cw_decomp_create(C.byref(g), C.byref(o), int(px), int(py), C.byref(self.h))
            _check(self.lib, None, rc, "cw_decomp_create")
            return
        idp = None
        if not loopback:
            if nccl_id is None or len(nccl_id) != 128:
                raise ValueError("nccl_id: the 128 bytes of nccl_unique_id, the same on every rank")
            idp = (C.c_ubyte * 128)(*nccl_id)
        rc = self.lib.cw_decomp_create_ranked(C.byref(g), C.byref(o), int(px), int(py), int(rank), int(nranks), idp,
                                              C.byref(self.h))
        _check(self.lib, None, rc, "cw_decomp_create_ranked")

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.cw_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()

    def upload_case(self, case):
        _check(self.lib, self.h, self.lib.cw_decomp_upload_case(self.h, case.h), "cw_decomp_upload_case")
        return self

    def step(self, n=1):
        _check(self.lib, self.h, self.lib.cw_step(self.h, n), "cw_step")

    def sync(self):
        _check(self.lib, self.h, self.lib.cw_sync(self.h), "cw_sync")

    def launches(self):
        v = C.c_longlong()
        self.lib.cw_launch_count(self.h, C.byref(v))
        return v.value

    def field(self, name, n=0):
        L = Layout()
        if self.lib.cw_layout_of(C.byref(self.g), C.byref(self.o), F[name], C.byref(L)) != 0:
            raise KeyError(name)
        out = np.empty(L.total, dtype=np.float64)
        rc = self.lib.cw_decomp_download(self.h, F[name], n, out.ctypes.data_as(C.POINTER(C.c_double)), out.size)
        _check(self.lib, self.h, rc, "cw_decomp_download")
        return out


class Batch:
    """Several domains of uneven sizes advanced together: every kernel launch covers all members
    (one handle, cw_batch_create). Members share the precision and the acoustic step count."""

    def __init__(self, grids, options, lib=None):
        self.lib = lib or capi.load()
        n = len(grids)
        self.grids, self.options = list(grids), list(options)
        ga = (Grid * n)(*grids)
        oa = (Options * n)(*options)
        self.h = C.c_void_p()
        rc = self.lib.cw_batch_create(n, ga, oa, C.byref(self.h))
        _check(self.lib, None, rc, "cw_batch_create")
        self.n = n

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.cw_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()

    def upload_case(self, member, case):
        _check(self.lib, self.h, self.lib.cw_member_upload_case(self.h, member, case.h), "cw_member_upload_case")
        return self

    def set_autotune(self, on=True):
        """The next six steps time the kernels' block shapes over all members; each kernel then keeps its fastest."""
        self.lib.cw_set_autotune(self.h, 1 if on else 0)
        return self

    def step(self, n=1):
        _check(self.lib, self.h, self.lib.cw_step(self.h, n), "cw_step")
        return self

    def sync(self):
        _check(self.lib, self.h, self.lib.cw_sync(self.h), "cw_sync")

    def launches(self):
        v = C.c_longlong()
        self.lib.cw_launch_count(self.h, C.byref(v))
        return v.value

    def diagnostics(self, member):
        """dyn::Diagnostics::compute of the current state (the diag.csv values, plus max_abs_q), as a dict."""
        d = capi.Diag()
        _check(self.lib, self.h, self.lib.cw_diagnostics(self.h, member, C.byref(d)), "cw_diagnostics")
        return d.as_dict()

    def snapshot(self, member, directory, step, time, q_names=None):
        """Writes directory/snap_<step>.{json,bin} in CPPWRF's snapshot format."""
        na = capi.names_array(q_names)
        rc = self.lib.cw_snapshot_write(self.h, member, str(directory).encode(), step, time, na[0] if na else None)
        if rc != 0:
            raise CwError(f"cw_snapshot_write: {self.lib.cw_output_last_error().decode()}")

    def layout(self, member, name, n=0):
        L = Layout()
        rc = self.lib.cw_member_field_layout(self.h, member, F[name], n, C.byref(L))
        _check(self.lib, self.h, rc, "cw_member_field_layout")
        return L

    def field(self, member, name, n=0):
        L = self.layout(member, name, n)
        out = np.empty(L.total, dtype=np.float64)
        rc = self.lib.cw_member_download(self.h, member, F[name], n, out.ctypes.data_as(C.POINTER(C.c_double)),
                                         out.size)
        _check(self.lib, self.h, rc, "cw_member_download")
        return out


class Server:
    """The served form (include/cw_serve.h): a C++ request loop on its own thread that admits requests by
    device-memory footprint, keeps them resident and advances them together in batched steps."""

    def __init__(self, budget_bytes=150e9, max_resident=256, precision=MIXED, device=0, keep_results=True, lib=None,
                 test_fail_creates=0):
        self.lib = lib or capi.load()
        cfg = capi.ServeConfig()
        self.lib.cw_serve_default_config(C.byref(cfg))
        cfg.hbm_budget_bytes, cfg.max_resident, cfg.precision = float(budget_bytes), int(max_resident), int(precision)
        cfg.device, cfg.keep_results = int(device), 1 if keep_results else 0
        cfg.test_fail_creates = int(test_fail_creates)
        self.h = C.c_void_p()
        rc = self.lib.cw_serve_create(C.byref(cfg), C.byref(self.h))
        if rc != 0:
            raise CwError(f"cw_serve_create failed ({rc})")
        self.cases = {}

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.cw_serve_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()

    def _err(self, what, rc):
        msg = self.lib.cw_serve_last_error(self.h)
        raise CwError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def submit(self, case, nsteps):
        rid = C.c_longlong()
        rc = self.lib.cw_serve_submit(self.h, case.h, int(nsteps), C.byref(rid))
        if rc != 0:
            self._err("cw_serve_submit", rc)
        self.cases[rid.value] = (case.g, case.o)
        return rid.value

    def wait(self, rid, seconds=-1.0):
        return self.lib.cw_serve_wait(self.h, rid, float(seconds))

    def drain(self):
        self.lib.cw_serve_drain(self.h)

    def result(self, rid, name, n=0):
        g, o = self.cases[rid]
        L = Layout()
        if self.lib.cw_layout_of(C.byref(g), C.byref(o), F[name], C.byref(L)) != 0:
            raise KeyError(name)
        out = np.empty(L.total, dtype=np.float64)
        rc = self.lib.cw_serve_result(self.h, rid, F[name], n, out.ctypes.data_as(C.POINTER(C.c_double)), out.size)
        if rc != 0:
            self._err("cw_serve_result", rc)
        return out

    def latency(self, rid):
        v = C.c_double()
        if self.lib.cw_serve_latency(self.h, rid, C.byref(v)) != 0:
            self._err("cw_serve_latency", -1)
        return v.value

    def release(self, rid):
        self.lib.cw_serve_release(self.h, rid)

    def stats(self):
        st = capi.ServeStats()
        self.lib.cw_serve_stats_get(self.h, C.byref(st))
        return {k: getattr(st, k) for k, _ in capi.ServeStats._fields_}
