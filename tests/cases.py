# SPDX-License-Identifier: GPL-3.0-or-later
"""Case definitions shared by the tests: the reference's regression configurations and small variants."""
import json
import os

from cppwrf_b200 import capi

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "reference_snapshots.json")))
KINDS = {"straka": capi.STRAKA, "warm_bubble": capi.WARM_BUBBLE, "igw": capi.IGW, "rest_state": capi.REST_STATE,
         "squall2d": capi.SQUALL2D}
BCS = {"periodic": capi.PERIODIC, "symmetric": capi.SYMMETRIC, "open": capi.OPEN}


def ideal_case(cfg, lib=None, u0=None, **opt):
    """A capi.Case of an ideal configuration dict (tests/golden/reference_snapshots.json style)."""
    g = capi.grid(cfg["nx"], cfg["ny"], cfg["nz"], cfg["dx"], cfg["dt"], cfg["ztop"], dy=cfg["dy"],
                  bc_x=BCS[cfg["bc_x"]], bc_y=BCS[cfg["bc_y"]])
    o = capi.default_options(lib, khdif=cfg["khdif"], kvdif=cfg["kvdif"], pr_inv=cfg["pr_inv"])
    o.diff_opt = 1 if (cfg["khdif"] > 0 or cfg["kvdif"] > 0) else 0
    o.n_moist = cfg.get("n_moist", 0)
    o.n_scalars = cfg.get("n_scalars", o.n_moist)
    o.mp_physics = cfg.get("mp_physics", 0)
    for k, v in opt.items():
        setattr(o, k, v)
    kw = {} if u0 is None else {"u0": u0}
    return capi.Case(g, o, lib).gen_ideal(KINDS[cfg["kind"]], **kw)


def golden_config(name):
    return dict(GOLDEN["cases"][name]["config"])


def lam_case(nx=24, ny=20, nz=14, seed=3, n_moist=5, n_scalars=5, diff=False, hybrid_opt=2, precision=capi.FP64,
             bc=(capi.SPECIFIED, capi.SPECIFIED), mapped=False):
    """A limited-area case (terrain, hybrid coordinate, moist species, specified boundaries) from a seed; bc = the
    (x, y) boundary kinds (open or periodic sides take no boundary data)."""
    g = capi.grid(nx, ny, nz, 15000.0, 90.0, 0.0, dy=15000.0, p_top=5000.0, bc_x=bc[0], bc_y=bc[1])
    o = capi.default_options(None, flat=0, n_moist=n_moist, n_scalars=n_scalars,
                             lbc=int(capi.SPECIFIED in bc), time_step_sound=4, precision=precision,
                             mapped=int(mapped))
    if diff:
        o.diff_opt, o.khdif, o.kvdif, o.pr_inv = 1, 3000.0, 1.0, 3.0
    return capi.Case(g, o).gen_lam(seed=seed, hybrid_opt=hybrid_opt)


# small variants for quick parity runs (same physics as the goldens, fewer points)
SMALL = {
    "straka_small": dict(golden_config("straka"), nx=64, nz=32, ztop=3200.0, run_time=3.0),
    "warm_bubble_small": dict(golden_config("warm_bubble"), nx=48, nz=40, ztop=4000.0, run_time=3.0),
    "igw_small": dict(golden_config("igw"), nx=60, run_time=18.0),
    "rest_state_small": dict(golden_config("rest_state"), nx=12, ny=10, nz=16, run_time=30.0),
}


def with_coriolis(case, f=1.0e-4, e=5.0e-5, sina=0.2, cosa=0.98):
    """Turn on the Coriolis terms (BaseState::coriolis) with uniform f, e and a rotated grid (sina, cosa)."""
    for name, value in (("F", f), ("E", e), ("SINA", sina), ("COSA", cosa)):
        a, _ = case.field(name)
        a[:] = value
    case.o.coriolis = 1
    return case


def with_map_factors(case, amp=0.02):
    """Horizontally varying map factors, f, e and grid rotation (a case made with mapped=True): smooth seeded
    patterns over every stored point, halos included; msfvx_inv = 1 / msfvx."""
    import numpy as np
    base = {"MSFTX": 1.0, "MSFTY": 1.01, "MSFUX": 1.0, "MSFUY": 1.01, "MSFVX": 1.0, "MSFVY": 1.01, "F": 1.0e-4,
            "E": 5.0e-5, "SINA": 0.1, "COSA": 0.99}
    for n, (name, b) in enumerate(base.items()):
        a, _ = case.field(name)
        x = np.arange(a.size, dtype=np.float64)
        a[:] = b * (1.0 + amp * np.sin(0.013 * x + 0.7 * n))
    inv, _ = case.field("MSFVX_INV")
    vx, _ = case.field("MSFVX")
    inv[:] = 1.0 / vx
    return case


def every_option_case():
    """A LAM case with every option the path accepts on at once (their interactions): varying map factors with
    Coriolis, km_opt 4 with damp_opt 1, the flux-limited sixth-order filter, hypsometric_opt 2, w_damping."""
    case = with_map_factors(lam_case(seed=31, diff=True, mapped=True))
    case.o.km_opt, case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 4, 1, 8000.0, 0.2
    case.o.diff_6th_opt, case.o.diff_6th_factor, case.o.hypsometric_opt, case.o.w_damping = 2, 0.12, 2, 1
    return case
