# SPDX-License-Identifier: GPL-3.0-or-later
"""cw_upload_fields / cw_download_fields (several fields, one synchronisation) move the same bytes as the per-field
cw_upload / cw_download, in the FP64 and the mixed form, and a step between them sees the uploaded state."""
import ctypes as C

import numpy as np
import pytest

from cppwrf_b200 import Domain, capi
from cases import lam_case

pytestmark = pytest.mark.gpu

NAMES = ["U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL"]


@pytest.mark.parametrize("prec", [capi.FP64, capi.MIXED], ids=["fp64", "mixed"])
def test_fields_round_trip_and_step(prec):
    case = lam_case(seed=27, precision=prec)
    a = Domain(case.g, case.o).upload_case(case)
    b = Domain(case.g, case.o).upload_case(case)
    lib = a.lib
    items = [(capi.F[n], 0) for n in NAMES] + [(capi.F["Q_2"], q) for q in range(case.o.n_scalars)]
    host = [a.field(n) + 0.0 for n in NAMES] + [a.field("Q_2", q) + 0.0 for q in range(case.o.n_scalars)]
    for x in host:  # a perturbation both handles receive, one through each entry point
        x *= 1.0 + 1e-6
    nf = len(items)
    fields = (C.c_int * nf)(*[f for f, _ in items])
    ns = (C.c_int * nf)(*[q for _, q in items])
    ptrs = (C.POINTER(C.c_double) * nf)(*[x.ctypes.data_as(C.POINTER(C.c_double)) for x in host])
    counts = (C.c_size_t * nf)(*[x.size for x in host])
    assert lib.cw_upload_fields(a.h, 0, nf, fields, ns, ptrs, counts) == 0
    for (f, q), x in zip(items, host):
        assert lib.cw_upload(b.h, f, q, x.ctypes.data_as(C.POINTER(C.c_double)), x.size) == 0
    a.step(2)
    b.step(2)
    outs = [np.empty_like(x) for x in host]
    optr = (C.POINTER(C.c_double) * nf)(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in outs])
    assert lib.cw_download_fields(a.h, 0, nf, fields, ns, optr, counts) == 0
    for (f, q), o, name in zip(items, outs, NAMES + [f"Q_2[{q}]" for q in range(case.o.n_scalars)]):
        ref = np.empty_like(o)
        assert lib.cw_download(b.h, f, q, ref.ctypes.data_as(C.POINTER(C.c_double)), ref.size) == 0
        assert np.array_equal(o.view(np.uint64), ref.view(np.uint64)), name
    bad_counts = (C.c_size_t * nf)(*([host[0].size + 1] + [x.size for x in host[1:]]))
    assert lib.cw_download_fields(a.h, 0, nf, fields, ns, optr, bad_counts) != 0  # a wrong count is refused


def window_mask(L):
    """The points of a field's allocation inside its window (its domain and halo)."""
    if L.uniform:
        return np.ones(L.total, dtype=bool)
    k = np.arange(L.nz if L.rank == 3 else 1, dtype=np.int64)[:, None, None]
    j = np.arange(L.wj0, L.wj1, dtype=np.int64)[None, :, None]
    i = np.arange(L.wi0, L.wi1, dtype=np.int64)[None, None, :]
    m = np.zeros(L.total, dtype=bool)
    m[(L.offset + i + j * L.sj + k * L.sk).ravel()] = True
    return m


@pytest.mark.parametrize("prec", [capi.FP64, capi.MIXED], ids=["fp64", "mixed"])
def test_window_copies_equal_whole_copies(prec):
    """cw_upload_windows / cw_download_windows: the window points only; a step after them equals a step after whole
    copies bit for bit, the downloaded window points equal the whole download's, and the host padding is untouched."""
    case = lam_case(seed=29, precision=prec)
    a = Domain(case.g, case.o).upload_case(case)
    b = Domain(case.g, case.o).upload_case(case)
    lib = a.lib
    items = [(capi.F[n], 0) for n in NAMES] + [(capi.F["Q_2"], q) for q in range(case.o.n_scalars)]
    names = NAMES + ["Q_2"] * case.o.n_scalars
    host = [a.field(n, q) * (1.0 + 1e-6) for n, (_, q) in zip(names, items)]
    masks = [window_mask(a.layout(n, q)) for n, (_, q) in zip(names, items)]
    nf = len(items)
    fields = (C.c_int * nf)(*[f for f, _ in items])
    ns = (C.c_int * nf)(*[q for _, q in items])
    ptrs = (C.POINTER(C.c_double) * nf)(*[x.ctypes.data_as(C.POINTER(C.c_double)) for x in host])
    counts = (C.c_size_t * nf)(*[x.size for x in host])
    assert lib.cw_upload_windows(a.h, 0, nf, fields, ns, ptrs, counts) == 0
    assert lib.cw_upload_fields(b.h, 0, nf, fields, ns, ptrs, counts) == 0
    a.step(2)
    b.step(2)
    outs = [np.full_like(x, 7.0) for x in host]
    optr = (C.POINTER(C.c_double) * nf)(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in outs])
    assert lib.cw_download_windows(a.h, 0, nf, fields, ns, optr, counts) == 0
    refs = [np.empty_like(x) for x in host]
    rptr = (C.POINTER(C.c_double) * nf)(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in refs])
    assert lib.cw_download_fields(b.h, 0, nf, fields, ns, rptr, counts) == 0
    for o, r, m, name in zip(outs, refs, masks, names):
        assert np.array_equal(o[m].view(np.uint64), r[m].view(np.uint64)), name
        assert np.all(o[~m] == 7.0), name  # the padding is not written
