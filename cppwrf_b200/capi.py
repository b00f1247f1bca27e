# SPDX-License-Identifier: GPL-3.0-or-later
"""ctypes mirror of include/cw_dycore.h: the structures, field ids and the library loader.

The shared library is the product: libcw_dycore.so, built in-tree by cppwrf_b200/build.py (CUDA
sm_100a kernels + C++20 host code). Nothing here falls back to a CPU implementation: a missing
library raises, and every dynamics call goes to the device through the C ABI.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcw_dycore.so")

# enum cw_bc
PERIODIC, SYMMETRIC, SPECIFIED, OPEN = 0, 1, 2, 3
# enum cw_precision
FP64, MIXED = 0, 1
# enum cw_field
FIELDS = [
    "U_1", "U_2", "V_1", "V_2", "W_1", "W_2", "T_1", "T_2", "PH_1", "PH_2", "MU_1", "MU_2",
    "P", "AL", "ALT", "PHP", "WW", "MUT", "MUU", "MUV", "MUTS", "MUUS", "MUVS", "RU", "RV", "RW",
    "RU_M", "RV_M", "WW_M", "CQU", "CQV", "CQW", "H_DIABATIC",
    "RU_TEND", "RV_TEND", "RW_TEND", "T_TEND", "PH_TEND", "MU_TEND",
    "RU_TENDF", "RV_TENDF", "RW_TENDF", "T_TENDF", "PH_TENDF",
    "MUB", "PB", "ALB", "T_INIT", "QV_BASE", "PHB", "HT",
    "MSFTX", "MSFTY", "MSFUX", "MSFUY", "MSFVX", "MSFVY", "MSFVX_INV", "F", "E", "SINA", "COSA", "RAINNC", "RAINNCV",
    "Q_1", "Q_2", "Q_TENDF",
]
F = {name: n for n, name in enumerate(FIELDS)}
NFIELDS = len(FIELDS)
# the prognostic state a step updates (compared bit for bit by the parity tests)
STATE_FIELDS = ["U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL", "WW", "RU_M", "RV_M", "WW_M",
                "MUTS", "MUUS", "MUVS", "U_1", "V_1", "W_1", "T_1", "PH_1", "MU_1", "ALT", "PHP", "MUT",
                "MUU", "MUV", "RU", "RV", "RW"]
# enum cw_lbc_var / cw_lbc_side
LBC_U, LBC_V, LBC_T, LBC_PH, LBC_MU = range(5)
XS, XE, YS, YE = range(4)
# enum cw_ideal_kind
REST_STATE, STRAKA, WARM_BUBBLE, IGW, SQUALL2D = range(5)
DEFAULT = -1.0e300
# the fill points of one step (cw_decomp_plan)
(FILL_MU1, FILL_PREP0, FILL_PREP1, FILL_SS0, FILL_UV, FILL_AC, FILL_POST, FILL_FIN, FILL_Q1PD, FILL_SCPD, FILL_Q2,
 FILL_END_P, FILL_WS0, FILL_WS1, FILL_MP, FILL_MP_P, FILL_XK) = range(17)
# cw_decomp_plan's field numbers beyond the field ids
FID_W, FID_Q2, FID_Q1, FID_QSC = 1000, 2000, 3000, 4000
# cw_download_noalloc: scratch capacity (doubles) and return codes
NOALLOC_SCRATCH_DOUBLES = 1048576
NOALLOC_EBADARG, NOALLOC_ETOOBIG, NOALLOC_ECUDA = -1, -2, -3


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("dt", C.c_double), ("ztop", C.c_double), ("p_top", C.c_double), ("bc_x", C.c_int),
                ("bc_y", C.c_int)]


class Options(C.Structure):
    _fields_ = [("khdif", C.c_double), ("kvdif", C.c_double), ("pr_inv", C.c_double), ("top_lid", C.c_int),
                ("h_adv_order", C.c_int), ("v_adv_order", C.c_int), ("w_damping", C.c_int),
                ("w_crit_cfl", C.c_double), ("epssm", C.c_double), ("smdiv", C.c_double), ("emdiv", C.c_double),
                ("damp_opt", C.c_int), ("hypsometric_opt", C.c_int), ("zdamp", C.c_double),
                ("dampcoef", C.c_double), ("time_step_sound", C.c_int), ("moist_adv_opt", C.c_int),
                ("scalar_adv_opt", C.c_int), ("tke_adv_opt", C.c_int), ("diff_opt", C.c_int), ("km_opt", C.c_int),
                ("flat", C.c_int), ("n_moist", C.c_int), ("n_scalars", C.c_int), ("lbc", C.c_int),
                ("precision", C.c_int), ("mp_physics", C.c_int), ("mp_tend_lim", C.c_double),
                ("diff_6th_opt", C.c_int), ("diff_6th_factor", C.c_double), ("coriolis", C.c_int),
                ("mapped", C.c_int)]


_DP = C.POINTER(C.c_double)


class Vertical(C.Structure):
    _fields_ = [(n, _DP) for n in ("znu", "dnw", "rdnw", "c1h", "c2h", "c3h", "c4h", "znw", "dn", "rdn", "fnm",
                                   "fnp", "c1f", "c2f", "c3f", "c4f", "u_base", "v_base", "t_base",
                                   "qv_base_1d", "z_base")] + \
               [(n, C.c_double) for n in ("cf1", "cf2", "cf3", "cfn", "cfn1", "rdx", "rdy", "p_top", "t0")]


class Layout(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("rank", C.c_int), ("uniform", C.c_int),
                ("stagger", C.c_char), ("si", C.c_int64), ("sj", C.c_int64), ("sk", C.c_int64),
                ("offset", C.c_int64), ("total", C.c_int64), ("wi0", C.c_int), ("wi1", C.c_int),
                ("wj0", C.c_int), ("wj1", C.c_int)]


class IdealParams(C.Structure):
    _fields_ = [("kind", C.c_int)] + [(n, C.c_double) for n in (
        "theta0", "n_bv", "u0", "xc", "zc", "xr", "zr", "amplitude", "radius", "a", "p_surf")]


class LamParams(C.Structure):
    _fields_ = [("seed", C.c_uint64)] + [(n, C.c_double) for n in (
        "t_surf", "lapse", "t_strat", "p_surf", "hill_height", "hill_halfwidth", "orog_max", "u_mean", "u_pert",
        "rh_mean", "rh_pert", "q_patch_max", "theta_pert", "wind_pert", "etac")] + [("hybrid_opt", C.c_int)]


class ServeConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_double), ("max_resident", C.c_int), ("precision", C.c_int),
                ("device", C.c_int), ("keep_results", C.c_int), ("test_fail_creates", C.c_int)]


class ServeStats(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in ("submitted", "completed", "failed", "rejected", "ticks")] + \
               [(n, C.c_int) for n in ("resident", "pending", "max_resident_seen")] + \
               [(n, C.c_double) for n in ("used_bytes", "max_used_bytes", "p50_s", "p99_s", "mean_s", "max_s",
                                          "gp_steps", "wall_s", "gp_steps_per_s")]


# cw_diag (include/cw_output.h): dyn::DiagRow in the order of the diag.csv columns, then max_abs_q
DIAG_KEYS = ("max_abs_u", "max_abs_v", "max_abs_w", "min_th_pert", "max_th_pert", "dry_mass", "theta_mass",
             "total_energy", "max_abs_q")


class Diag(C.Structure):
    _fields_ = [(n, C.c_double) for n in DIAG_KEYS]

    def as_dict(self):
        return {n: getattr(self, n) for n in DIAG_KEYS}


class SnapshotFields(C.Structure):
    _fields_ = [(n, _DP) for n in ("u_2", "v_2", "w_2", "t_2", "p", "ph_2", "mu_2", "pb", "phb", "t_init", "mub")] + \
               [("q_2", C.POINTER(_DP)), ("rainnc", _DP), ("rainncv", _DP)]


_lib = None


def load(path=None):
    """Loads libcw_dycore.so (in-tree build) and declares its entry points."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(p)
    vp, ip, i, dp, sz = C.c_void_p, C.POINTER(C.c_int), C.c_int, _DP, C.c_size_t
    sig = {
        "cw_default_options": (i, [C.POINTER(Options)]),
        "cw_layout_of": (i, [C.POINTER(Grid), C.POINTER(Options), i, C.POINTER(Layout)]),
        "cw_case_create": (i, [C.POINTER(Grid), C.POINTER(Options), C.POINTER(vp)]),
        "cw_case_destroy": (i, [vp]),
        "cw_case_field": (i, [vp, i, i, C.POINTER(dp), C.POINTER(Layout)]),
        "cw_case_vertical": (i, [vp, C.POINTER(Vertical)]),
        "cw_case_lbc": (i, [vp, i, i, i, C.POINTER(dp), C.POINTER(dp), C.POINTER(sz)]),
        "cw_case_lbc_time": (i, [vp, dp]),
        "cw_default_ideal_params": (i, [C.POINTER(IdealParams), i]),
        "cw_gen_ideal": (i, [vp, C.POINTER(IdealParams)]),
        "cw_default_lam_params": (i, [C.POINTER(LamParams)]),
        "cw_gen_lam": (i, [vp, C.POINTER(LamParams)]),
        "cw_create": (i, [C.POINTER(Grid), C.POINTER(Options), C.POINTER(vp)]),
        "cw_destroy": (i, [vp]),
        "cw_set_vertical": (i, [vp, C.POINTER(Vertical)]),
        "cw_upload": (i, [vp, i, i, dp, sz]),
        "cw_download": (i, [vp, i, i, dp, sz]),
        "cw_field_layout": (i, [vp, i, i, C.POINTER(Layout)]),
        "cw_field_device_ptr": (i, [vp, i, i, C.POINTER(vp)]),
        "cw_set_lbc": (i, [vp, i, i, dp, dp, sz]),
        "cw_set_lbc_scalar": (i, [vp, i, i, dp, dp, sz]),
        "cw_set_lbc_time": (i, [vp, C.c_double]),
        "cw_step": (i, [vp, i]),
        "cw_set_dt": (i, [vp, C.c_double, i]),
        "cw_n_sound": (i, [vp, ip]),
        "cw_set_stream": (i, [vp, vp]),
        "cw_sync": (i, [vp]),
        "cw_selftest_wait": (i, [vp, C.c_longlong]),
        "cw_last_error": (C.c_char_p, [vp]),
        "cw_launch_count": (i, [vp, C.POINTER(C.c_longlong)]),
        "cw_upload_case": (i, [vp, vp]),
        "cw_member_upload_case": (i, [vp, i, vp]),
        "cw_profile": (i, [vp, i, ip]),
        "cw_profile_entry": (i, [vp, i, C.c_char_p, i, dp, C.POINTER(C.c_longlong)]),
        "cw_use_device": (i, [i]),
        "cw_set_graph": (i, [vp, i]),
        "cw_batch_create": (i, [i, C.POINTER(Grid), C.POINTER(Options), C.POINTER(vp)]),
        "cw_members": (i, [vp, ip]),
        "cw_member_upload": (i, [vp, i, i, i, dp, sz]),
        "cw_member_download": (i, [vp, i, i, i, dp, sz]),
        "cw_member_field_layout": (i, [vp, i, i, i, C.POINTER(Layout)]),
        "cw_download_noalloc": (i, [vp, i, i, dp, sz]),
        "cw_batch_add": (i, [vp, C.POINTER(Grid), C.POINTER(Options), ip]),
        "cw_batch_remove": (i, [vp, i]),
        "cw_batch_adopt": (i, [vp, vp, ip]),
        "cw_set_autotune": (i, [vp, i]),
        "cw_check_finite": (i, [vp, i, ip, ip, ip, ip, ip]),
        "cw_batch_release": (i, [vp, i, C.POINTER(vp)]),
        "cw_decomp_patch": (i, [C.POINTER(Grid), i, i, i, C.POINTER(C.c_int)]),
        "cw_decomp_create": (i, [C.POINTER(Grid), C.POINTER(Options), i, i, C.POINTER(vp)]),
        "cw_decomp_upload": (i, [vp, i, i, dp, sz]),
        "cw_decomp_download": (i, [vp, i, i, dp, sz]),
        "cw_decomp_upload_case": (i, [vp, vp]),
        "cw_nccl_unique_id": (i, [C.POINTER(C.c_ubyte)]),
        "cw_decomp_create_ranked": (i, [C.POINTER(Grid), C.POINTER(Options), i, i, i, i, C.POINTER(C.c_ubyte),
                                        C.POINTER(vp)]),
        "cw_decomp_plan": (i, [C.POINTER(Grid), C.POINTER(Options), i, i, i, i, i, ip, C.POINTER(C.c_longlong), i,
                               ip]),
        "cw_check_div_const": (i, [C.c_ulonglong, C.c_ulonglong, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
        "cw_autotune_choice": (i, [vp, C.c_char_p, ip]),
        "cw_footprint": (i, [C.POINTER(Grid), C.POINTER(Options), C.POINTER(sz)]),
        "cw_case_clone": (i, [vp, C.POINTER(vp)]),
        "cw_case_config": (i, [vp, C.POINTER(Grid), C.POINTER(Options)]),
        "cw_member_config": (i, [vp, i, C.POINTER(Grid), C.POINTER(Options)]),
        "cw_set_cfl_diagnostics": (i, [vp, i]),
        "cw_cfl_max": (i, [vp, i, dp, dp]),
        "cw_diagnostics": (i, [vp, i, C.POINTER(Diag)]),
        "cw_diag_header": (i, [C.c_char_p, sz]),
        "cw_diag_format_row": (i, [C.c_longlong, C.c_double, C.POINTER(Diag), C.c_double, C.c_char_p, sz]),
        "cw_snapshot_write_host": (i, [C.c_char_p, C.c_longlong, C.c_double, C.POINTER(Grid), C.POINTER(Options),
                                       C.POINTER(SnapshotFields), C.POINTER(C.c_char_p)]),
        "cw_snapshot_write": (i, [vp, i, C.c_char_p, C.c_longlong, C.c_double, C.POINTER(C.c_char_p)]),
        "cw_output_last_error": (C.c_char_p, []),
        "cw_serve_default_config": (i, [C.POINTER(ServeConfig)]),
        "cw_serve_create": (i, [C.POINTER(ServeConfig), C.POINTER(vp)]),
        "cw_serve_destroy": (i, [vp]),
        "cw_serve_submit": (i, [vp, vp, i, C.POINTER(C.c_longlong)]),
        "cw_serve_wait": (i, [vp, C.c_longlong, C.c_double]),
        "cw_serve_drain": (i, [vp]),
        "cw_serve_result": (i, [vp, C.c_longlong, i, i, dp, sz]),
        "cw_serve_latency": (i, [vp, C.c_longlong, dp]),
        "cw_serve_release": (i, [vp, C.c_longlong]),
        "cw_serve_stats_get": (i, [vp, C.POINTER(ServeStats)]),
        "cw_serve_last_error": (C.c_char_p, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name, None)
        if f is None:
            continue
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def diag_header(lib=None):
    """The diag.csv header line (io::DiagWriter)."""
    lib = lib or load()
    buf = C.create_string_buffer(512)
    if lib.cw_diag_header(buf, 512) < 0:
        raise RuntimeError("cw_diag_header")
    return buf.value.decode()


def diag_row(step, time, diag, wall_s, lib=None):
    """One diag.csv line (io::DiagWriter::row) of a cw_diag (a Diag or a dict of DIAG_KEYS)."""
    lib = lib or load()
    d = diag if isinstance(diag, Diag) else Diag(*[diag.get(k, 0.0) for k in DIAG_KEYS])
    buf = C.create_string_buffer(1024)
    if lib.cw_diag_format_row(step, time, C.byref(d), wall_s, buf, 1024) < 0:
        raise RuntimeError("cw_diag_format_row")
    return buf.value.decode()


def names_array(names):
    if names is None:
        return None
    arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
    return C.cast(arr, C.POINTER(C.c_char_p)), arr


def snapshot_write_host(directory, step, time, g, o, fields, q_fields=(), q_names=None, lib=None):
    """cw_snapshot_write_host over whole-allocation float64 arrays: fields = {"u_2": array, ..., "mub": array}."""
    lib = lib or load()
    keep = [np.ascontiguousarray(fields[n], dtype=np.float64) for n in
            ("u_2", "v_2", "w_2", "t_2", "p", "ph_2", "mu_2", "pb", "phb", "t_init", "mub")]
    qs = [np.ascontiguousarray(q, dtype=np.float64) for q in q_fields]
    qp = (_DP * max(1, len(qs)))(*[q.ctypes.data_as(_DP) for q in qs])
    rain = [np.ascontiguousarray(fields[n], dtype=np.float64) if n in fields else None for n in ("rainnc", "rainncv")]
    f = SnapshotFields(*[a.ctypes.data_as(_DP) for a in keep], C.cast(qp, C.POINTER(_DP)),
                       *[r.ctypes.data_as(_DP) if r is not None else None for r in rain])
    na = names_array(q_names)
    rc = lib.cw_snapshot_write_host(str(directory).encode(), step, time, C.byref(g), C.byref(o), C.byref(f),
                                    na[0] if na else None)
    if rc != 0:
        raise RuntimeError(lib.cw_output_last_error().decode())


def default_options(lib=None, **kw):
    lib = lib or load()
    o = Options()
    lib.cw_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def grid(nx, ny, nz, dx, dt, ztop=0.0, dy=None, p_top=0.0, bc_x=PERIODIC, bc_y=PERIODIC):
    return Grid(nx, ny, nz, dx, dx if dy is None else dy, dt, ztop, p_top, bc_x, bc_y)


def as_array(ptr, n, owner=None):
    """A numpy view of n doubles at a C pointer (no copy); the view keeps `owner` (the object whose
    destruction frees the memory) alive."""
    if n == 0:
        return np.zeros(0)
    buf = (C.c_double * n).from_address(C.addressof(ptr.contents))
    buf._owner = owner
    return np.frombuffer(buf, dtype=np.float64)


class Case:
    """A host-side input set (cw_case) of one domain."""

    def __init__(self, g, o, lib=None):
        self.lib = lib or load()
        self.h = C.c_void_p()
        rc = self.lib.cw_case_create(C.byref(g), C.byref(o), C.byref(self.h))
        if rc != 0:
            raise ValueError(f"cw_case_create failed ({rc})")
        self.g, self.o = g, o

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.cw_case_destroy(self.h)
            self.h = C.c_void_p()

    def field(self, name, n=0):
        """(array view of the whole allocation, Layout) of a field."""
        p, L = _DP(), Layout()
        rc = self.lib.cw_case_field(self.h, F[name], n, C.byref(p), C.byref(L))
        if rc != 0:
            raise KeyError(name)
        return as_array(p, L.total, self), L

    def vertical(self):
        v = Vertical()
        self.lib.cw_case_vertical(self.h, C.byref(v))
        return v

    def lbc(self, var, side, scalar=False):
        vals, tends, cnt = _DP(), _DP(), C.c_size_t()
        rc = self.lib.cw_case_lbc(self.h, 1 if scalar else 0, var, side, C.byref(vals), C.byref(tends), C.byref(cnt))
        if rc != 0:
            return None
        return as_array(vals, cnt.value, self), as_array(tends, cnt.value, self)

    def lbc_time(self):
        t = C.c_double()
        self.lib.cw_case_lbc_time(self.h, C.byref(t))
        return t.value

    def gen_ideal(self, kind, **kw):
        p = IdealParams()
        self.lib.cw_default_ideal_params(C.byref(p), kind)
        for k, v in kw.items():
            setattr(p, k, v)
        rc = self.lib.cw_gen_ideal(self.h, C.byref(p))
        if rc != 0:
            raise RuntimeError(f"cw_gen_ideal failed ({rc})")
        # the generator sets p_top from the sounding
        self.g.p_top = self.vertical().p_top
        return self

    def gen_lam(self, **kw):
        p = LamParams()
        self.lib.cw_default_lam_params(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        rc = self.lib.cw_gen_lam(self.h, C.byref(p))
        if rc != 0:
            raise RuntimeError(f"cw_gen_lam failed ({rc})")
        self.g.p_top = self.vertical().p_top
        return self


def layout_index(L, i, j, k):
    return L.offset + i * L.si + j * L.sj + k * L.sk


def interior(arr, L):
    """The logical points (k, j, i) of a field array (no halo), as a new array."""
    k = np.arange(L.nz)[:, None, None]
    j = np.arange(L.ny)[None, :, None]
    i = np.arange(L.nx)[None, None, :]
    return arr[L.offset + i * L.si + j * L.sj + k * L.sk]
