# SPDX-License-Identifier: GPL-3.0-or-later
"""Properties the reference's unit tests pin (tests/unit/test_scalars.cpp, test_large_step.cpp), on the GPU
path: a constant tracer stays constant, the PD limiter keeps a tracer non-negative where plain advection
undershoots, tracer mass is conserved without diffusion, a rest state stays at rest, repeated runs are
bit-identical."""
import numpy as np
import pytest

import cases
from cppwrf_b200 import Domain, capi
from cases import lam_case

pytestmark = pytest.mark.gpu


def tracer_case(adv, khdif=75.0, n_scalars=2):
    """The small Straka case (periodic x-z) with passive tracers: species 0 = 1 everywhere, species 1 a blob."""
    cfg = dict(cases.SMALL["straka_small"], khdif=khdif, kvdif=khdif)
    case = cases.ideal_case(cfg, n_moist=0, n_scalars=n_scalars, scalar_adv_opt=adv)
    for which in ("Q_1", "Q_2"):
        for n in range(n_scalars):
            q, L = case.field(which, n)
            q[:] = 1.0 if (n == 0 and n_scalars > 1) else 0.0
        q, L = case.field(which, n_scalars - 1)
        for k in range(L.nz):
            for i in range(-3, L.nx + 3):
                x, z = i - 20, k - 8
                q[L.offset + i * L.si + k * L.sk] = max(0.0, 1.0 - (x * x / 36 + z * z / 16))
    return case


def run(case, steps):
    d = Domain(case.g, case.o).upload_case(case)
    d.step(steps)
    return d


def q_interior(d, n):
    return capi.interior(d.field("Q_2", n), d.layout("Q_2", n))


def test_constant_tracer_stays_constant():
    d = run(tracer_case(adv=1), 60)
    assert np.abs(q_interior(d, 0) - 1.0).max() < 1e-12


def test_pd_keeps_tracer_nonnegative_where_plain_advection_undershoots():
    pd = q_interior(run(tracer_case(adv=1), 60), 1)
    plain = q_interior(run(tracer_case(adv=0), 60), 1)
    assert pd.min() >= -1e-12 * pd.max()
    assert plain.min() < -1e-9  # the limiter is doing something


def test_tracer_mass_conserved_without_diffusion():
    case = tracer_case(adv=1, khdif=0.0, n_scalars=1)
    v, nz = case.vertical(), case.g.nz
    c1h = np.ctypeslib.as_array(v.c1h, shape=(nz,)).copy()
    c2h = np.ctypeslib.as_array(v.c2h, shape=(nz,)).copy()
    dnw = np.ctypeslib.as_array(v.dnw, shape=(nz,)).copy()

    def mass(d):
        q = q_interior(d, 0)
        mt = (capi.interior(d.field("MUB"), d.layout("MUB")) + capi.interior(d.field("MU_2"), d.layout("MU_2")))[0]
        m = c1h[:, None, None] * mt[None] + c2h[:, None, None]
        return float(np.sum(m * q * (-dnw)[:, None, None]))

    d = Domain(case.g, case.o).upload_case(case)
    m0 = mass(d)
    d.step(60)
    assert abs(mass(d) - m0) <= 1e-13 * abs(m0)


def test_rest_state_stays_at_rest():
    d = run(cases.ideal_case(cases.SMALL["rest_state_small"]), 10)
    for name in ("U_2", "V_2", "MU_2"):
        assert np.all(capi.interior(d.field(name), d.layout(name)) == 0.0), name
    assert np.abs(capi.interior(d.field("W_2"), d.layout("W_2"))).max() < 1e-9


def test_repeated_runs_bit_identical():
    case = lam_case(nx=33, ny=27, nz=15, seed=17, diff=True)
    a, b = run(case, 4), run(case, 4)
    for name in capi.STATE_FIELDS:
        assert np.array_equal(a.field(name).view(np.uint64), b.field(name).view(np.uint64)), name


def test_inertial_oscillation():
    """Coriolis on an f-plane (the reference's dycore check 2, configs/inertial.ini): a uniform u0 = 10 m/s with
    f = 1e-3 1/s and no pressure gradient turns as u = u0 cos(f t), v = -u0 sin(f t); within 1e-3 m/s over one
    period, checked every quarter period."""
    cfg = dict(cases.golden_config("rest_state"), nx=8, ny=8, nz=20, dx=2000.0, dy=2000.0, ztop=20000.0, dt=10.0,
               khdif=0.0, kvdif=0.0)
    case = cases.with_coriolis(cases.ideal_case(cfg, u0=10.0), f=1.0e-3, e=0.0, sina=0.0, cosa=1.0)
    d = Domain(case.g, case.o).upload_case(case)
    worst = 0.0
    for n in range(1, 5):
        d.step(157)
        t = 1570.0 * n
        u = capi.interior(d.field("U_2"), d.layout("U_2"))
        v = capi.interior(d.field("V_2"), d.layout("V_2"))
        worst = max(worst, float(np.abs(u - 10.0 * np.cos(1.0e-3 * t)).max()),
                    float(np.abs(v + 10.0 * np.sin(1.0e-3 * t)).max()))
    assert worst <= 1.0e-3, worst


def test_map_factor_invariance_bit_exact():
    """The map-factor form is invariant (the reference's dycore check 1): squall2d (moist, Kessler, PD advection)
    with a constant map factor m = 2 and dx = 2000 m equals m = 1 and dx = 1000 m bit for bit -- every scaling by 2
    is exact in floating point. emdiv = 0: the external-mode filter uses the grid dx."""
    from test_oracle_properties import scaled_pair
    a, b = scaled_pair()
    da, db = run(a, 20), run(b, 20)
    names = ["U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL", "RAINNC"]
    for name in names:
        assert np.array_equal(da.field(name).view(np.uint64), db.field(name).view(np.uint64)), name
    for n in range(a.o.n_scalars):
        assert np.array_equal(da.field("Q_2", n).view(np.uint64), db.field("Q_2", n).view(np.uint64)), n
