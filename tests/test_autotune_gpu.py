# SPDX-License-Identifier: GPL-3.0-or-later
"""Block-shape autotuning: the tuning steps are ordinary steps and every shape computes the same values, so an
autotuned run is bit-identical to a run with the default shapes; afterwards each tunable kernel has a choice. A
column kernel's shape is its warps per column block (8, 16 or 4): only the parallel loops over levels change."""
import numpy as np
import pytest

from cppwrf_b200 import Batch, Domain, capi
from cases import lam_case

pytestmark = pytest.mark.gpu

TUNABLE = ["k_tend", "k_tendf_rk1", "k_uv", "k_q_march", "k_q_face_pd", "k_q_scale_pd", "k_q_update_pd",
           "k_ls_prep", "k_ss_prep", "k_ac", "k_finish"]  # k_q_march: levels per block; the last four: warps per
#                                                             column block


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED], ids=["fp64", "mixed"])
def test_autotuned_equals_default(precision):
    case = lam_case(nx=37, ny=29, nz=16, seed=13, diff=True, precision=precision)
    a = Domain(case.g, case.o).upload_case(case).set_autotune(True)
    b = Domain(case.g, case.o).upload_case(case)
    assert a.autotune_choice("k_tend") == -1
    a.step(4)  # four of the six tuning steps
    a.step(4)  # the last two, then two graph-replayed steps with the chosen shapes
    b.step(8)
    for name in capi.STATE_FIELDS:
        assert np.array_equal(a.field(name).view(np.uint64), b.field(name).view(np.uint64)), name
    for n in range(case.o.n_scalars):
        assert np.array_equal(a.field("Q_2", n).view(np.uint64), b.field("Q_2", n).view(np.uint64)), n
    for k in TUNABLE:
        assert a.autotune_choice(k) in (0, 1, 2), k


def test_autotuned_batch_equals_default():
    cases = [lam_case(nx=20 + 3 * m, ny=16 + m, nz=12, seed=40 + m) for m in range(3)]
    a = Batch([c.g for c in cases], [c.o for c in cases]).set_autotune(True)
    b = Batch([c.g for c in cases], [c.o for c in cases])
    for m, c in enumerate(cases):
        a.upload_case(m, c)
        b.upload_case(m, c)
    a.step(4)
    b.step(4)
    for m in range(len(cases)):
        for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P"):
            assert np.array_equal(a.field(m, name).view(np.uint64), b.field(m, name).view(np.uint64)), (m, name)
