# SPDX-License-Identifier: GPL-3.0-or-later
"""Pins the oracle against the reference's own CPU FP64 dycore compiled from its sources (oracle/_ref), on
the paths the regression goldens do not reach: terrain, the hybrid coordinate, moist species with the
positive-definite limiter, specified lateral boundaries (relaxation, spec zone, flow-dependent scalars),
constant-K diffusion in 3-D, symmetric walls in 3-D. Both sides take pow from cw_pow (the reference
through symbol interposition), so the comparison is bit for bit. Runs only where the reference sources
are present (this build's container); the fixtures in tests/golden keep the pin on other machines."""
import numpy as np
import pytest

import _oracle
import _refpath  # noqa: F401
import refdump as _refdump
import cases
from cases import lam_case
from cppwrf_b200 import capi

pytestmark = pytest.mark.skipif(not _refdump.available(), reason="reference sources / oracle/_ref not present")


def compare(orc, ref, case):
    bad = []
    for name in [n for n in capi.FIELDS if not n.startswith("Q_")]:
        a = orc.array(name)
        b = ref[name]
        if b.size == 0:
            continue
        if not np.array_equal(a.view(np.uint64), b.view(np.uint64)):
            d = np.nonzero(a.view(np.uint64) != b.view(np.uint64))[0]
            bad.append(f"{name}: {d.size} differ, first {d[0]}: oracle {a[d[0]]!r} ref {b[d[0]]!r}")
    for n in range(case.o.n_scalars):
        for name in ("Q_1", "Q_2", "Q_TENDF"):
            a, b = orc.array(name, n), ref[f"{name}:{n}"]
            if not np.array_equal(a.view(np.uint64), b.view(np.uint64)):
                d = np.nonzero(a.view(np.uint64) != b.view(np.uint64))[0]
                bad.append(f"{name}[{n}]: {d.size} differ, first {d[0]}: oracle {a[d[0]]!r} ref {b[d[0]]!r}")
    return bad


@pytest.mark.parametrize("kw", [dict(), dict(diff=True), dict(hybrid_opt=0, seed=5), dict(n_moist=2, n_scalars=3)],
                         ids=["lam", "lam_diffusion", "lam_sigma", "lam_tracer"])
def test_oracle_equals_reference_lam(kw):
    case = lam_case(**kw)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


def test_oracle_equals_reference_3d_symmetric_diffusion():
    cfg = dict(cases.golden_config("rest_state"), nx=14, ny=12, nz=12, bc_x="symmetric", bc_y="symmetric",
               khdif=200.0, kvdif=5.0, run_time=40.0)
    case = cases.ideal_case(cfg, u0=3.0)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(4)
    ref = _refdump.run(case, 4, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


def test_oracle_equals_reference_default_glibc_pow():
    """The oracle with glibc's pow (lane rule) against the unmodified reference build."""
    cfg = dict(cases.SMALL["straka_small"])
    case = cases.ideal_case(cfg)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=False)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("own", [True, False], ids=["cw_pow_cw_sin", "glibc"])
def test_oracle_equals_reference_w_rayleigh_damping(own):
    """damp_opt 3 (advance_w's implicit Rayleigh damping of w in the upper 8 km): with our pow and sin in both,
    and with glibc's in both."""
    case = lam_case(seed=7)
    case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 3, 8000.0, 0.2
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN if own else _oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=own)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)
    plain = lam_case(seed=7)
    undamped = _oracle.Oracle(plain, pow_mode=_oracle.POW_OWN if own else _oracle.POW_GLIBC)
    undamped.step(3)
    assert not np.array_equal(orc.array("W_2"), undamped.array("W_2"))  # the damping acted


@pytest.mark.parametrize("opt,diff", [(1, False), (2, True)], ids=["linear", "flux_limited_with_k"])
def test_oracle_equals_reference_sixth_order_filter(opt, diff):
    """diff_6th_opt 1 / 2: the sixth-order horizontal filter of the first RK stage (dynamics and every scalar), alone
    and after constant-K diffusion, on a LAM case (specified boundaries: the filter skips three rows)."""
    case = lam_case(seed=9, diff=diff)
    case.o.diff_6th_opt, case.o.diff_6th_factor = opt, 0.12
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


def test_oracle_equals_reference_sixth_order_periodic_2d():
    cfg = dict(cases.SMALL["straka_small"])
    case = cases.ideal_case(cfg, diff_6th_opt=2, diff_6th_factor=0.25)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=False)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("own", [True, False], ids=["cw_sin", "glibc"])
def test_oracle_equals_reference_rayleigh_damping_to_base_state(own):
    """damp_opt 2: the first stage's Rayleigh damping of u, v, w, theta toward the base-state profile in the upper
    8 km (libmvec's sin on the lanes of the reference's vectorised level loops in the glibc build)."""
    case = lam_case(seed=11)
    case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 2, 8000.0, 0.003
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN if own else _oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=own)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


def test_oracle_equals_reference_rayleigh_damping_2d():
    cfg = dict(cases.SMALL["igw_small"])
    case = cases.ideal_case(cfg, damp_opt=2, zdamp=4000.0, dampcoef=0.01)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=False)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("own", [True, False], ids=["cw_log", "glibc"])
def test_oracle_equals_reference_hypsometric_log_pressure(own):
    """hypsometric_opt 2: calc_p_rho_phi's inverse density from the geopotential thickness over the log of the
    layer's pressure ratio (libmvec's log on the lanes of the reference's i loop in the glibc build, on the whole
    domain and on the interior after the boundary update)."""
    case = lam_case(seed=15)
    case.o.hypsometric_opt = 2
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN if own else _oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=own)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)
    linear = lam_case(seed=15)
    lin = _oracle.Oracle(linear, pow_mode=_oracle.POW_OWN if own else _oracle.POW_GLIBC)
    lin.step(3)
    assert not np.array_equal(orc.array("AL"), lin.array("AL"))


def test_oracle_equals_reference_hypsometric_log_pressure_2d():
    cfg = dict(cases.SMALL["igw_small"])
    case = cases.ideal_case(cfg, hypsometric_opt=2)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=False)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("bc,kw", [((capi.OPEN, capi.OPEN), dict()), ((capi.OPEN, capi.OPEN), dict(diff=True)),
                                   ((capi.OPEN, capi.PERIODIC), dict(n_moist=2, n_scalars=3)),
                                   ((capi.PERIODIC, capi.OPEN), dict(hybrid_opt=0))],
                         ids=["open", "open_diffusion", "open_x_periodic_y", "periodic_x_open_y"])
def test_oracle_equals_reference_open_boundaries(bc, kw):
    """Open lateral boundaries (WRF open_xs/xe/ys/ye): the radiation condition on the boundary faces of u and v, the
    open terms of the outermost cells' advection (u, v, w, theta, geopotential, every scalar, PD at rk 3), the
    boundary faces' acoustic update and time sums, the diffusion's loop limits; corners where both are open."""
    case = lam_case(seed=17, bc=bc, **kw)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


def test_oracle_equals_reference_open_sixth_order_2d():
    """2-D x-z with open x (squall-line style) and the sixth-order filter's open-side limits."""
    cfg = dict(cases.SMALL["warm_bubble_small"], bc_x="open")
    case = cases.ideal_case(cfg, diff_6th_opt=2, diff_6th_factor=0.12)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=False)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("own", [True, False], ids=["cw_cos", "glibc"])
def test_oracle_equals_reference_eddy_viscosity_damping(own):
    """damp_opt 1 (cal_dampkm): the horizontal eddy viscosities of constant-K diffusion raised toward ds^2/dt in the
    upper 8 km of the columns inside the boundary zone (libmvec's cos on the lanes of the reference's column loop
    in the glibc build)."""
    case = lam_case(seed=19, diff=True)
    case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 1, 8000.0, 0.2
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN if own else _oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=own)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)
    plain = lam_case(seed=19, diff=True)
    undamped = _oracle.Oracle(plain, pow_mode=_oracle.POW_OWN if own else _oracle.POW_GLIBC)
    undamped.step(3)
    assert not np.array_equal(orc.array("U_2"), undamped.array("U_2"))  # the damping acted


def test_oracle_equals_reference_eddy_viscosity_damping_2d():
    cfg = dict(cases.SMALL["straka_small"])
    case = cases.ideal_case(cfg, damp_opt=1, zdamp=1500.0, dampcoef=0.2)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=False)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("bc,damp", [((capi.SPECIFIED, capi.SPECIFIED), 0), ((capi.OPEN, capi.OPEN), 0),
                                     ((capi.OPEN, capi.PERIODIC), 0), ((capi.SPECIFIED, capi.SPECIFIED), 1)],
                         ids=["lam", "open", "open_x_periodic_y", "lam_dampkm"])
def test_oracle_equals_reference_smagorinsky_2d(bc, damp):
    """diff_opt 1 with km_opt 4: the horizontal eddy viscosities from the 2-D deformation (Smagorinsky, c_s 0.25) with
    the terrain-following metric terms, the boundary faces' copies and the zero outermost rows of specified boundaries
    (and with damp_opt 1 on top)."""
    case = lam_case(seed=21, diff=True, bc=bc)
    case.o.km_opt = 4
    if damp:
        case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 1, 8000.0, 0.2
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


def test_oracle_equals_reference_smagorinsky_2d_xz():
    case = cases.ideal_case(dict(cases.SMALL["straka_small"]), km_opt=4)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=False)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("kw", [dict(), dict(bc=(capi.OPEN, capi.PERIODIC), n_moist=2, n_scalars=3)],
                         ids=["lam", "open_x_periodic_y"])
def test_oracle_equals_reference_coriolis(kw):
    """BaseState::coriolis: the Coriolis terms of the u, v, w tendencies with uniform f, e and a rotated grid."""
    case = cases.with_coriolis(lam_case(seed=23, **kw))
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)
    plain = lam_case(seed=23, **kw)
    still = _oracle.Oracle(plain, pow_mode=_oracle.POW_OWN)
    still.step(3)
    assert not np.array_equal(orc.array("V_2"), still.array("V_2"))  # the terms acted


@pytest.mark.parametrize("kw", [dict(), dict(diff=True)], ids=["lam", "lam_diffusion"])
def test_oracle_equals_reference_mapped(kw):
    """BaseState::mapped: horizontally varying map factors, f, e, sina, cosa (2-D storage), the Coriolis terms and the
    curvature terms from the map factors' gradients, in every term that carries a map factor."""
    case = cases.with_map_factors(lam_case(seed=25, mapped=True, **kw))
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


def test_oracle_equals_reference_every_option():
    """Every option the path accepts on at once (cases.every_option_case), for their interactions."""
    case = cases.every_option_case()
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)
