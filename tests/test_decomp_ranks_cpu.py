# SPDX-License-Identifier: GPL-3.0-or-later
"""A domain's patches over ranks (cw_decomp_create_ranked; tiles_mpi.cpp:35-64, docs/MPI.md section 3) on CPU: the
plan of the exchange between ranks (cw_decomp_plan, no device) carried out by gloo ranks. Each rank packs the boxes
it sends from its own patches, the segments cross as point-to-point messages, each rank unpacks what it receives and
copies between its own patches; afterwards every point of every patch's window inside the domain holds the owner's
value -- the plan misses no point, the two ranks of a pair list the same boxes in the same order, and every box lands
where it belongs. The device side of the same plan (packing and unpacking kernels, loopback transport) is
tests/test_decomp_gpu.py's."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from cppwrf_b200 import capi, decomp_plan  # noqa: E402

SETS = {"prep0+q2": [capi.FILL_PREP0, capi.FILL_Q2], "prep1": [capi.FILL_PREP1], "uv": [capi.FILL_UV],
        "post": [capi.FILL_POST], "fin": [capi.FILL_FIN], "ws": [capi.FILL_WS0, capi.FILL_WS1]}


def setup(nx=30, ny=24, nz=4, kind="lam"):
    if kind == "2d":  # an x-z slice with symmetric walls (no y exchange; rows of stride 0)
        g = capi.grid(nx, 1, nz, 1000.0, 5.0, 6000.0, bc_x=capi.SYMMETRIC, bc_y=capi.PERIODIC)
        o = capi.default_options(None, n_moist=1, n_scalars=1, time_step_sound=4)
        return g, o
    if kind == "open":
        g = capi.grid(nx, ny, nz, 15000.0, 90.0, 0.0, dy=15000.0, p_top=5000.0, bc_x=capi.OPEN, bc_y=capi.SYMMETRIC)
        o = capi.default_options(None, flat=0, n_moist=2, n_scalars=2, lbc=0, time_step_sound=4)
        return g, o
    g = capi.grid(nx, ny, nz, 15000.0, 90.0, 0.0, dy=15000.0, p_top=5000.0, bc_x=capi.SPECIFIED, bc_y=capi.SPECIFIED)
    o = capi.default_options(None, flat=0, n_moist=2, n_scalars=2, lbc=1, time_step_sound=4)
    return g, o


def layout(g, o, fid):
    name = "Q_2" if fid >= capi.FID_Q2 else capi.FIELDS[fid]
    L = capi.Layout()
    assert capi.load().cw_layout_of(g, o, capi.F[name], L) == 0
    return L


def patch_box(g, px, py, t):
    import ctypes as C
    box = (C.c_int * 4)()
    assert capi.load().cw_decomp_patch(g, px, py, t, box) == 0
    return tuple(box)


def geometry(g, L, p):
    """A patch's window of a field and the points it owns (the rule of cw_decomp_create's layouts: the patch and a
    halo of 3, the east / north edge patches up to the field's staggered extent)."""
    i0, i1, j0, j1 = p
    s = L.stagger.decode() if isinstance(L.stagger, bytes) else chr(L.stagger)
    win = (i0 - 3, (L.nx if i1 == g.nx else i1) + 3, j0 - 3, (L.ny if j1 == g.ny else j1) + 3)
    own = (i0, g.nx + 1 if (s == "U" and i1 == g.nx) else i1, j0, g.ny + 1 if (s == "V" and j1 == g.ny) else j1)
    return win, own


def value(fid, i, j, k):
    return fid * 1.0e6 + k * 1.0e4 + (j + 5) * 100.0 + (i + 5)


def exchange(rank, world, px, py, sets, send, recv, kind="lam"):
    """The fill point on this rank; send(peer, array) / recv(peer, n) the transport. Returns the points left wrong."""
    g, o = setup(kind=kind)
    plan = decomp_plan(g, o, px, py, rank, world, sets)
    fids = sorted({int(f) for r in range(world) for f in decomp_plan(g, o, px, py, r, world, sets)[:, 4]})
    assert fids, "no box crosses between ranks"
    mine = [t for t in range(px * py) if t % world == rank]
    boxes = {t: patch_box(g, px, py, t) for t in range(px * py)}
    data = {}
    for t in mine:
        for f in fids:
            L = layout(g, o, f)
            (wi0, wi1, wj0, wj1), (oi0, oi1, oj0, oj1) = geometry(g, L, boxes[t])
            a = np.full((L.nz, wj1 - wj0, wi1 - wi0), np.nan)
            for j in range(max(wj0, oj0), min(wj1, oj1)):
                for i in range(max(wi0, oi0), min(wi1, oi1)):
                    a[:, j - wj0, i - wi0] = [value(f, i, j, k) for k in range(L.nz)]
            data[t, f] = (a, wi0, wj0)

    def view(t, f, i0, i1, j0, j1, nk):
        a, wi0, wj0 = data[t, f]
        return a[:nk, j0 - wj0:j1 - wj0, i0 - wi0:i1 - wi0]

    # pack: the segment of each receiving rank, boxes in offset order, points i fastest, then j, then k
    sent = plan[plan[:, 0] == 0]
    n_send = int(max((b[10] + (b[6] - b[5]) * (b[8] - b[7]) * b[9] for b in sent), default=0))
    sbuf = np.full(n_send, np.nan)
    for role, peer, me, t, f, i0, i1, j0, j1, nk, off in sent:
        assert t in mine and me not in mine and peer == me % world
        v = view(t, f, i0, i1, j0, j1, nk)
        assert not np.isnan(v).any(), "a packed point is not the owner's"
        sbuf[off:off + v.size] = v.ravel()
    got = plan[plan[:, 0] == 1]
    n_recv = int(max((b[10] + (b[6] - b[5]) * (b[8] - b[7]) * b[9] for b in got), default=0))
    rbuf = np.full(n_recv, np.nan)
    for q in range(world):  # lower ranks first on both sides: every pair's two messages in one order
        if q == rank:
            continue
        for direction in ((0, 1) if rank < q else (1, 0)):
            rows = sent if direction == 0 else got
            seg = rows[rows[:, 1] == q]
            if not len(seg):
                continue
            lo = int(seg[0][10])
            hi = int(seg[-1][10] + (seg[-1][6] - seg[-1][5]) * (seg[-1][8] - seg[-1][7]) * seg[-1][9])
            assert np.all(np.diff(seg[:, 10]) > 0), "a segment's boxes out of order"
            if direction == 0:
                send(q, sbuf[lo:hi])
            else:
                rbuf[lo:hi] = recv(q, hi - lo)
    for role, peer, me, t, f, i0, i1, j0, j1, nk, off in got:
        assert me in mine and t not in mine and peer == t % world
        v = view(me, f, i0, i1, j0, j1, nk)
        v[...] = rbuf[off:off + v.size].reshape(v.shape)
    # the exchange between this rank's own patches (direct copies)
    for me in mine:
        for t in mine:
            if t == me:
                continue
            for f in fids:
                L = layout(g, o, f)
                (wi0, wi1, wj0, wj1), _ = geometry(g, L, boxes[me])
                _, (oi0, oi1, oj0, oj1) = geometry(g, L, boxes[t])
                i0, i1, j0, j1 = max(wi0, oi0), min(wi1, oi1), max(wj0, oj0), min(wj1, oj1)
                if i0 < i1 and j0 < j1:
                    view(me, f, i0, i1, j0, j1, L.nz)[...] = view(t, f, i0, i1, j0, j1, L.nz)
    # every window point inside the domain: the owner's value
    wrong = 0
    for (t, f), (a, wi0, wj0) in data.items():
        L = layout(g, o, f)
        for k in range(L.nz):
            for jj in range(a.shape[1]):
                for ii in range(a.shape[2]):
                    i, j = ii + wi0, jj + wj0
                    if 0 <= i < L.nx and 0 <= j < L.ny and a[k, jj, ii] != value(f, i, j, k):
                        wrong += 1
    return wrong, len(sent), len(got)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, px, py, q, kind="lam"):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))

    def send(peer, a):
        dist.send(torch.from_numpy(np.ascontiguousarray(a)), dst=peer)

    def recv(peer, n):
        t = torch.empty(n, dtype=torch.float64)
        dist.recv(t, src=peer)
        return t.numpy()

    out = {}
    for name, sets in SETS.items():
        out[name] = exchange(rank, world, px, py, sets, send, recv, kind)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


@pytest.mark.parametrize("px,py,world,kind", [(2, 1, 2, "lam"), (2, 2, 2, "lam"), (3, 2, 3, "lam"), (3, 1, 3, "2d"),
                                              (2, 2, 4, "open")])
def test_exchange_between_ranks_fills_every_halo_point(px, py, world, kind):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, px, py, q, kind)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        for name, (wrong, n_sent, n_got) in res[r].items():
            assert wrong == 0, (r, name, wrong)
            assert n_sent > 0 and n_got > 0, (r, name)


def test_both_ranks_of_a_pair_list_the_same_boxes():
    """What rank p packs for rank r is, box for box and offset for offset within the segment, what r unpacks."""
    g, o = setup()
    for px, py, world in ((2, 2, 2), (3, 2, 3), (3, 2, 6)):
        for sets in SETS.values():
            plans = [decomp_plan(g, o, px, py, r, world, sets) for r in range(world)]
            for p in range(world):
                for r in range(world):
                    if p == r:
                        continue
                    s = plans[p][(plans[p][:, 0] == 0) & (plans[p][:, 1] == r)]
                    d = plans[r][(plans[r][:, 0] == 1) & (plans[r][:, 1] == p)]
                    assert s.shape == d.shape
                    if len(s):
                        assert np.array_equal(s[:, 2:10], d[:, 2:10])
                        assert np.array_equal(s[:, 10] - s[0, 10], d[:, 10] - d[0, 10])


def test_one_rank_has_no_boxes_between_ranks():
    g, o = setup()
    assert len(decomp_plan(g, o, 3, 2, 0, 1, [capi.FILL_FIN])) == 0


def test_plan_refuses_bad_ranks_and_fill_points():
    g, o = setup()
    for rank, world, sets in ((2, 2, [capi.FILL_FIN]), (0, 5, [capi.FILL_FIN]), (-1, 2, [capi.FILL_FIN]),
                              (0, 2, [99])):
        with pytest.raises(RuntimeError):
            decomp_plan(g, o, 2, 2, rank, world, sets)
