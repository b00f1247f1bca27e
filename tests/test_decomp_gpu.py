# SPDX-License-Identifier: GPL-3.0-or-later
"""One domain decomposed into px x py patches (cw_decomp_create, CPPWRF's tile decomposition: src/core/tiles.hpp,
docs/MPI.md section 3): each patch computes only the points it owns, in fields allocated for its patch and a halo of
3 and indexed with the domain's indices, and at every fill point receives the points of its halo that other
patches own before the domain's boundary fill. After the same steps, every field gathered from the patches equals
the undecomposed domain's bit for bit -- halos and the domain's lateral halos included."""
import numpy as np
import pytest

import cases
from cases import lam_case
from cppwrf_b200 import Decomp, Domain, capi

pytestmark = pytest.mark.gpu


def window(L):
    """The points of a field's allocation inside its window (the domain and its halo; the row padding and the
    leading pad hold no point of the field: a gathered field has 0 there, as tile::download gives it)."""
    if L.uniform:
        return np.ones(L.total, dtype=bool)
    k = np.arange(L.nz, dtype=np.int64)[:, None, None]
    j = np.arange(L.wj0, L.wj1, dtype=np.int64)[None, :, None]
    i = np.arange(L.wi0, L.wi1, dtype=np.int64)[None, None, :]
    m = np.zeros(L.total, dtype=bool)
    m[(L.offset + i + j * L.sj + k * L.sk).ravel()] = True
    return m


def compare(dec, dom, case):
    bad = []
    names = [(n, 0) for n in capi.FIELDS if not n.startswith("Q_")]
    names += [(q, s) for s in range(case.o.n_scalars) for q in ("Q_1", "Q_2", "Q_TENDF")]
    for name, n in names:
        w = window(dom.layout(name, n))
        a, b = np.where(w, dec.field(name, n), 0.0), np.where(w, dom.field(name, n), 0.0)
        if not np.array_equal(a.view(np.uint64), b.view(np.uint64)):
            d = np.nonzero(a.view(np.uint64) != b.view(np.uint64))[0]
            L = dom.layout(name, n)
            k, r = divmod(int(d[0]) - L.offset, L.sk) if L.sk else (0, int(d[0]) - L.offset)
            j, i = divmod(r, L.sj) if L.sj else (0, r)
            bad.append(f"{name}[{n}]: {d.size} differ, first at (i {i}, j {j}, k {k}): decomposed {a[d[0]]!r} "
                       f"whole {b[d[0]]!r}")
    return bad


def run_both(case, px, py, nsteps, **ranks):
    dom = Domain(case.g, case.o).upload_case(case)
    dec = Decomp(case.g, case.o, px, py, **ranks).upload_case(case)
    dom.step(nsteps)
    dec.step(nsteps)
    dom.sync()
    dec.sync()
    return dec, dom


@pytest.mark.parametrize("px,py", [(2, 1), (1, 2), (2, 2), (3, 2)])
def test_lam_patches_equal_whole_domain(px, py):
    """Terrain, hybrid coordinate, 5 moist species with the PD limiter, specified boundaries (relaxation, spec zone,
    spec_bdy_final), 4 steps."""
    case = lam_case(nx=40, ny=34, nz=14, seed=71)
    dec, dom = run_both(case, px, py, 4)
    bad = compare(dec, dom, case)
    assert not bad, "\n".join(bad)


def test_lam_with_every_option_on_patches():
    """Varying map factors with Coriolis, km_opt 4 with damp_opt 1, the flux-limited sixth-order filter,
    hypsometric_opt 2 and w_damping, on 2 x 2 patches."""
    case = cases.every_option_case()
    dec, dom = run_both(case, 2, 2, 3)
    bad = compare(dec, dom, case)
    assert not bad, "\n".join(bad)


def test_open_boundaries_on_patches():
    case = lam_case(nx=36, ny=30, nz=12, seed=73, bc=(capi.OPEN, capi.OPEN))
    dec, dom = run_both(case, 2, 2, 3)
    bad = compare(dec, dom, case)
    assert not bad, "\n".join(bad)


def test_2d_symmetric_split_along_x():
    """A 2-D x-z case with symmetric walls (warm bubble) on 3 patches along x."""
    case = cases.ideal_case(cases.SMALL["warm_bubble_small"])
    dec, dom = run_both(case, 3, 1, 3)
    bad = compare(dec, dom, case)
    assert not bad, "\n".join(bad)


def test_benchmark_workload_on_six_patches_mixed_and_fp64():
    """The 119 x 89 x 44 workload on 3 x 2 patches, in both forms (the mixed form is deterministic too)."""
    import bench
    for prec in (capi.FP64, capi.MIXED):
        case = bench.make_case(capi, prec)
        dec, dom = run_both(case, 3, 2, 2)
        bad = compare(dec, dom, case)
        assert not bad, "\n".join(bad)


@pytest.mark.parametrize("px,py,nranks", [(2, 1, 2), (2, 2, 4), (3, 2, 2), (3, 2, 6)])
def test_patches_over_ranks_loopback_equal_whole_domain(px, py, nranks):
    """cw_decomp_create_ranked in its loopback form: this process holds every patch, and the exchanges between patches
    of different ranks (t % nranks) go through the packing kernel, the packed send and receive buffers (a device copy
    in place of the NCCL transfer) and the unpacking kernel -- the ranks' path on one GPU but NCCL itself."""
    case = lam_case(nx=40, ny=34, nz=14, seed=71)
    dec, dom = run_both(case, px, py, 4, nranks=nranks, loopback=True)
    bad = compare(dec, dom, case)
    assert not bad, "\n".join(bad)


def test_benchmark_workload_over_three_ranks_loopback_mixed_and_fp64():
    import bench
    for prec in (capi.FP64, capi.MIXED):
        case = bench.make_case(capi, prec)
        dec, dom = run_both(case, 3, 2, 2, nranks=3, loopback=True)
        bad = compare(dec, dom, case)
        assert not bad, "\n".join(bad)


def test_every_option_over_ranks_loopback():
    case = cases.every_option_case()
    dec, dom = run_both(case, 2, 2, 3, nranks=2, loopback=True)
    bad = compare(dec, dom, case)
    assert not bad, "\n".join(bad)
