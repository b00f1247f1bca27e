# SPDX-License-Identifier: GPL-3.0-or-later
"""Parity of the CUDA FP64 path with the oracle: after N steps every field of the State, Tendencies and
BaseState (whole allocations, halos included) is bit-identical (tolerance 0). Both sides use cw_pow in
calc_p_rho_phi (the oracle in its interposed mode)."""
import numpy as np
import pytest

import _oracle
import cases
from cases import lam_case
from cppwrf_b200 import Domain, capi

pytestmark = pytest.mark.gpu


def compare_all(dom, orc, case, names=None):
    bad = []
    for name in names or [n for n in capi.FIELDS if not n.startswith("Q_")]:
        a = dom.field(name)
        b = orc.array(name)
        if not np.array_equal(a.view(np.uint64), b.view(np.uint64)):
            d = np.nonzero(a.view(np.uint64) != b.view(np.uint64))[0]
            bad.append(f"{name}: {d.size} differ, first at {d[0]}: gpu {a[d[0]]!r} oracle {b[d[0]]!r}")
    for n in range(case.o.n_scalars):
        for name in ("Q_1", "Q_2", "Q_TENDF"):
            a, b = dom.field(name, n), orc.array(name, n)
            if not np.array_equal(a.view(np.uint64), b.view(np.uint64)):
                d = np.nonzero(a.view(np.uint64) != b.view(np.uint64))[0]
                bad.append(f"{name}[{n}]: {d.size} differ, first at {d[0]}: gpu {a[d[0]]!r} oracle {b[d[0]]!r}")
    return bad


def run_pair(case, nsteps):
    dom = Domain(case.g, case.o).upload_case(case)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    dom.step(nsteps)
    dom.sync()
    orc.step(nsteps)
    return dom, orc


@pytest.mark.parametrize("name", sorted(cases.SMALL))
def test_ideal_small_bit_exact(name):
    cfg = cases.SMALL[name]
    case = cases.ideal_case(cfg)
    n = int(round(cfg["run_time"] / cfg["dt"]))
    dom, orc = run_pair(case, n)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("name", ["straka", "warm_bubble", "igw", "rest_state"])
def test_reference_regression_cases_bit_exact(name):
    cfg = cases.golden_config(name)
    case = cases.ideal_case(cfg)
    dom, orc = run_pair(case, int(round(cfg["run_time"] / cfg["dt"])))
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_graph_and_eager_identical():
    cfg = cases.SMALL["straka_small"]
    case = cases.ideal_case(cfg)
    a = Domain(case.g, case.o).upload_case(case)
    b = Domain(case.g, case.o).upload_case(case)
    b.set_graph(False)
    a.step(2)
    b.step(2)
    for name in ("U_2", "W_2", "T_2", "PH_2", "MU_2", "P"):
        assert np.array_equal(a.field(name), b.field(name)), name


@pytest.mark.parametrize("kw", [dict(), dict(diff=True), dict(hybrid_opt=0, seed=5), dict(n_moist=2, n_scalars=3),
                                dict(n_moist=0, n_scalars=0)],
                         ids=["lam", "lam_diffusion", "lam_sigma", "lam_tracer", "lam_dry"])
def test_lam_bit_exact(kw):
    """Terrain, hybrid coordinate, moist species (PD limiter at rk 3), specified boundaries (relaxation,
    spec zone, flow-dependent scalars), 4 steps."""
    case = lam_case(**kw)
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_lam_w_rayleigh_damping_bit_exact():
    """damp_opt 3: advance_w's implicit Rayleigh damping of w in the upper 8 km (sin = cw_sin on both sides)."""
    case = lam_case(seed=7)
    case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 3, 8000.0, 0.2
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("opt,diff", [(1, False), (2, True)], ids=["linear", "flux_limited_with_k"])
def test_lam_sixth_order_filter_bit_exact(opt, diff):
    """diff_6th_opt 1 / 2: the sixth-order horizontal filter (dynamics and scalars) at the first RK stage."""
    case = lam_case(seed=9, diff=diff)
    case.o.diff_6th_opt, case.o.diff_6th_factor = opt, 0.12
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_periodic_2d_sixth_order_filter_bit_exact():
    case = cases.ideal_case(dict(cases.SMALL["straka_small"]), diff_6th_opt=2, diff_6th_factor=0.25)
    dom, orc = run_pair(case, 3)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_lam_rayleigh_damping_to_base_state_bit_exact():
    """damp_opt 2: u, v, w, theta damped toward the base-state profile in the upper 8 km at the first stage."""
    case = lam_case(seed=11)
    case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 2, 8000.0, 0.003
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_2d_rayleigh_damping_bit_exact():
    case = cases.ideal_case(dict(cases.SMALL["igw_small"]), damp_opt=2, zdamp=4000.0, dampcoef=0.01)
    dom, orc = run_pair(case, 3)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_lam_hypsometric_log_pressure_bit_exact():
    """hypsometric_opt 2: calc_p_rho_phi's inverse density from the geopotential thickness over the log of the
    layer's pressure ratio (log = cw_log on both sides), on the whole domain and on the interior."""
    case = lam_case(seed=15)
    case.o.hypsometric_opt = 2
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_2d_hypsometric_log_pressure_bit_exact():
    case = cases.ideal_case(dict(cases.SMALL["igw_small"]), hypsometric_opt=2)
    dom, orc = run_pair(case, 3)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("bc,kw", [((capi.OPEN, capi.OPEN), dict()), ((capi.OPEN, capi.OPEN), dict(diff=True)),
                                   ((capi.OPEN, capi.PERIODIC), dict(n_moist=2, n_scalars=3)),
                                   ((capi.PERIODIC, capi.OPEN), dict(hybrid_opt=0))],
                         ids=["open", "open_diffusion", "open_x_periodic_y", "periodic_x_open_y"])
def test_lam_open_boundaries_bit_exact(bc, kw):
    """Open lateral boundaries: radiation on the boundary faces of u and v, the open terms of the outermost cells
    (u, v, w, theta, geopotential, every scalar incl. PD at rk 3), the faces' acoustic update and time sums, the
    diffusion's loop limits; 4 steps."""
    case = lam_case(seed=17, bc=bc, **kw)
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_2d_open_x_sixth_order_bit_exact():
    case = cases.ideal_case(dict(cases.SMALL["warm_bubble_small"], bc_x="open"), diff_6th_opt=2, diff_6th_factor=0.12)
    dom, orc = run_pair(case, 3)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_lam_eddy_viscosity_damping_bit_exact():
    """damp_opt 1: cal_dampkm's horizontal eddy viscosities near the top (cos = cw_cos on both sides) in the
    constant-K diffusion of the first stage, dynamics and scalars."""
    case = lam_case(seed=19, diff=True)
    case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 1, 8000.0, 0.2
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_2d_eddy_viscosity_damping_bit_exact():
    case = cases.ideal_case(dict(cases.SMALL["straka_small"]), damp_opt=1, zdamp=1500.0, dampcoef=0.2)
    dom, orc = run_pair(case, 3)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("bc,damp", [((capi.SPECIFIED, capi.SPECIFIED), 0), ((capi.OPEN, capi.OPEN), 0),
                                     ((capi.OPEN, capi.PERIODIC), 0), ((capi.SPECIFIED, capi.SPECIFIED), 1)],
                         ids=["lam", "open", "open_x_periodic_y", "lam_dampkm"])
def test_lam_smagorinsky_2d_bit_exact(bc, damp):
    """diff_opt 1 with km_opt 4: the 2-D Smagorinsky eddy viscosities from the deformation (metric terms, edge copies,
    zero outermost rows), with and without damp_opt 1 on top; 4 steps."""
    case = lam_case(seed=21, diff=True, bc=bc)
    case.o.km_opt = 4
    if damp:
        case.o.damp_opt, case.o.zdamp, case.o.dampcoef = 1, 8000.0, 0.2
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_2d_smagorinsky_bit_exact():
    case = cases.ideal_case(dict(cases.SMALL["straka_small"]), km_opt=4)
    dom, orc = run_pair(case, 3)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("kw", [dict(), dict(bc=(capi.OPEN, capi.PERIODIC), n_moist=2, n_scalars=3)],
                         ids=["lam", "open_x_periodic_y"])
def test_lam_coriolis_bit_exact(kw):
    """The Coriolis terms (uniform f, e, sina, cosa) of the u, v, w tendencies; 4 steps."""
    case = cases.with_coriolis(lam_case(seed=23, **kw))
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("kw", [dict(), dict(diff=True)], ids=["lam", "lam_diffusion"])
def test_lam_mapped_bit_exact(kw):
    """Horizontally varying map factors, f, e, sina, cosa: Coriolis and curvature terms and every map factor of the
    step; 4 steps."""
    case = cases.with_map_factors(lam_case(seed=25, mapped=True, **kw))
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_lam_every_option_bit_exact():
    """Every option the path accepts on at once (cases.every_option_case), for their interactions."""
    case = cases.every_option_case()
    dom, orc = run_pair(case, 4)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_cfl_maxima_equal_oracle():
    """LargeStep::cfl_max of every RK stage (the adaptive time step's input): the device maxima equal the oracle's,
    and recording them changes no field."""
    case = lam_case(seed=13)
    dom = Domain(case.g, case.o).upload_case(case).set_cfl_diagnostics()
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    for _ in range(2):
        dom.step(2)
        orc.step(2)
        got, want = dom.cfl_max(), orc.cfl_max()
        assert got == want, (got, want)
        assert all(v > 0 and h > 0 for v, h in got)
    bad = compare_all(dom, orc, case)
    assert not bad, "\n".join(bad)


def test_benchmark_workload_bit_exact():
    """The benchmark's 119 x 89 x 44 workload (bench.py), 2 steps."""
    import bench
    case = bench.make_case(capi, capi.FP64)
    dom, orc = run_pair(case, 2)
    bad = compare_all(dom, orc, case, names=capi.STATE_FIELDS)
    assert not bad, "\n".join(bad)


def test_launch_count_gates_the_plain_scalar_update():
    """At rk 3 the plain scalar update runs only when some species is not PD: a case whose species are all PD
    takes one launch less per step than the same case with one plain tracer (the count of the step's launches,
    the same graph or eager)."""
    pd = lam_case(n_moist=2, n_scalars=2)
    mixed = lam_case(n_moist=2, n_scalars=3)
    pd.o.scalar_adv_opt = mixed.o.scalar_adv_opt = 0  # the third species of `mixed` is a plain tracer
    assert pd.o.moist_adv_opt == 1 and mixed.o.moist_adv_opt == 1
    counts = []
    for case in (pd, mixed):
        dom = Domain(case.g, case.o).upload_case(case)
        dom.step(1)
        dom.sync()
        counts.append(dom.launches())
    assert counts[1] == counts[0] + 1, counts


def test_launches_per_step_of_the_lam_workload():
    """One step of the 119 x 89 x 44 workload in one CUDA graph: 72 launches in FP64 (the large-step tendencies as
    two launches, (u, v) and (w, phi, theta, mu)), 69 in the mixed form (one)."""
    import bench
    for prec, want in ((capi.FP64, 72), (capi.MIXED, 69)):
        case = bench.make_case(capi, prec)
        dom = Domain(case.g, case.o).upload_case(case)
        dom.step(1)  # the captured step
        dom.step(1)  # a replay: the count of the last call
        dom.sync()
        assert dom.launches() == want, (prec, dom.launches())
