# SPDX-License-Identifier: GPL-3.0-or-later
"""The served form: requests admitted by device-memory footprint into a running batch (continuous
batching), each result identical to the same request run alone, the budget never exceeded."""
import ctypes as C
import time

import numpy as np
import pytest

from cppwrf_b200 import Domain, Server, capi
from cases import lam_case

pytestmark = pytest.mark.gpu

FIELDS = ["U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL"]


def footprint(case):
    lib = capi.load()
    b = C.c_size_t()
    assert lib.cw_footprint(C.byref(case.g), C.byref(case.o), C.byref(b)) == 0
    return b.value


def check_alone(srv, rid, case, nsteps):
    alone = Domain(case.g, case.o).upload_case(case)
    alone.step(nsteps)
    for name in FIELDS:
        assert np.array_equal(srv.result(rid, name).view(np.uint64), alone.field(name).view(np.uint64)), (rid, name)
    for n in range(case.o.n_scalars):
        assert np.array_equal(srv.result(rid, "Q_2", n).view(np.uint64), alone.field("Q_2", n).view(np.uint64)), (rid, n)


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED], ids=["fp64", "mixed"])
def test_served_results_equal_alone(precision):
    spec = [(24, 20, 14, 3, 6), (31, 17, 14, 4, 9), (18, 26, 14, 5, 4), (40, 33, 14, 6, 7), (22, 18, 12, 8, 5)]
    cases = [lam_case(nx=nx, ny=ny, nz=nz, seed=s, precision=precision) for nx, ny, nz, s, _ in spec]
    fp = sorted(footprint(c) for c in cases)
    budget = fp[-1] + fp[-2]  # room for the two largest at once
    srv = Server(budget_bytes=budget, max_resident=4, precision=precision)
    ids = []
    for k, (c, sp) in enumerate(zip(cases, spec)):
        ids.append(srv.submit(c, sp[4]))
        if k == 1:
            time.sleep(0.05)  # the rest arrive while the first ones run
    srv.drain()
    st = srv.stats()
    assert st["completed"] == len(spec) and st["failed"] == 0, st
    assert st["max_used_bytes"] <= budget, st
    assert st["max_resident_seen"] >= 2, st
    assert 0 < st["p50_s"] <= st["p99_s"], st
    for rid, c, sp in zip(ids, cases, spec):
        check_alone(srv, rid, c, sp[4])
        assert srv.latency(rid) > 0
    srv.close()


def test_served_rejects_a_request_larger_than_the_budget():
    c = lam_case(nx=24, ny=20, nz=14, seed=3)
    srv = Server(budget_bytes=footprint(c) // 2, precision=capi.FP64)
    with pytest.raises(Exception):
        srv.submit(c, 3)
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_served_failed_batch_creation_does_not_block_later_requests():
    """A failure injected on the host into the first batch-handle creation (the test hook of cw_serve_config) fails
    only the request that needed it: the batch is not left half-made, and later requests of the same acoustic step
    count make a new one and complete, equal to the same requests alone."""
    cases = [lam_case(nx=24, ny=20, nz=14, seed=s) for s in (51, 52, 53)]
    srv = Server(budget_bytes=1e12, precision=capi.FP64, test_fail_creates=1)
    first = srv.submit(cases[0], 3)
    assert srv.wait(first) == -2  # failed: the injected creation error
    later = [srv.submit(c, 4) for c in cases[1:]]
    srv.drain()
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 2, st
    assert st["used_bytes"] == 0 and st["resident"] == 0, st
    for rid, c in zip(later, cases[1:]):
        check_alone(srv, rid, c, 4)
    srv.close()


def test_served_rejects_requests_without_steps():
    c = lam_case(nx=24, ny=20, nz=14, seed=3)
    srv = Server(budget_bytes=1e12, precision=capi.FP64)
    with pytest.raises(Exception):
        srv.submit(c, 0)
    st = srv.stats()
    assert st["submitted"] == 0 and st["failed"] == 0, st
    srv.close()
