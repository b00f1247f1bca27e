# SPDX-License-Identifier: GPL-3.0-or-later
"""Pins of the oracle against the reference's own CPU FP64 build (oracle/_ref, compiled from its sources) on the
benchmark configurations as they are stated, every field bit for bit:

- the 3-D limited-area workload (119 x 89 x 44, dx 15 km, dt 90 s, 4 acoustic substeps, hybrid coordinate,
  terrain, 5 moist species with the PD limiter at rk 3, specified boundaries), 3 steps, pow interposed by cw_pow
  on both sides (ref_harness_own, the oracle's OWN mode);
- the 2-D density current (Straka: 256 x 1 x 64, dx = dz = 100 m, dt 1 s, 6 acoustic substeps, K = 75 m^2/s,
  cold bubble of -15 K at x = 0, z = 3 km) over its whole 900 s, with glibc's pow and libmvec's lanes on both
  sides (the unmodified reference build, ref_harness, and the oracle's GLIBC mode).

CPU only; skipped where neither the reference sources nor oracle/_ref are present."""
import numpy as np
import pytest

import _oracle
import _refpath  # noqa: F401
import refdump as _refdump
import cases
from cppwrf_b200 import capi

pytestmark = pytest.mark.skipif(not _refdump.available(), reason="reference sources / oracle/_ref not present")


def straka_config1():
    """The 2-D density current of the first benchmark configuration (WRF's 257 x 3 x 65 staggered points)."""
    return dict(cases.golden_config("straka"), nx=256, run_time=900.0)


def compare(orc, ref, case):
    bad = []
    for name in [n for n in capi.FIELDS if not n.startswith("Q_")]:
        a, b = orc.array(name), ref[name]
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


def test_oracle_equals_reference_benchmark_workload():
    import bench
    case = bench.make_case(capi, capi.FP64)
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_OWN)
    orc.step(3)
    ref = _refdump.run(case, 3, own_pow=True)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


def test_oracle_glibc_equals_reference_density_current_900s():
    cfg = straka_config1()
    case = cases.ideal_case(cfg)
    assert case.g.nx == 256 and case.g.ny == 1 and case.g.nz == 64
    n = int(round(cfg["run_time"] / cfg["dt"]))
    orc = _oracle.Oracle(case, pow_mode=_oracle.POW_GLIBC)
    orc.step(n)
    ref = _refdump.run(case, n, own_pow=False)
    bad = compare(orc, ref, case)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("nsteps", [0, 2])
def test_harness_generated_lam_input_equals_written_input(nsteps):
    """ref_harness --lam (the case generated inside the harness, as the benchmark's reference arm runs it) gives
    every field bit for bit as the same case written by refdump.write_input: at step 0 (the input itself) and
    after 2 steps (the vertical arrays and boundary slabs too)."""
    w = dict(nx=30, ny=24, nz=16, dx=15000.0, dt=90.0, time_step_sound=4, p_top=5000.0, n_moist=5, hybrid_opt=2,
             etac=0.2)
    import bench
    case = bench.make_case(capi, capi.FP64, seed=4, w=w)
    a = _refdump.run(case, nsteps, own_pow=False)
    b = _refdump.run_lam(w, 4, nsteps)
    assert a.keys() == b.keys()
    bad = [k for k in a if not np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64))]
    assert not bad, bad
