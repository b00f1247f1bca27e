# SPDX-License-Identifier: GPL-3.0-or-later
"""The N > 1 path of bench.py on CPU (gloo, world size 2): every rank owns its own domain (a different seed,
different inputs), the job time is the maximum over ranks, the value is all ranks' points over that time,
and the reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from cppwrf_b200 import capi
    ms = 10.0 + 5.0 * rank  # the ranks' device times differ
    job_ms = bench.max_over_ranks(ms, world, "cpu")
    case = bench.make_case(capi, capi.FP64, seed=bench.shard_seed(rank),
                           w=dict(nx=16, ny=12, nz=10))  # a small domain of the same generator
    t, _ = case.field("T_2")
    import hashlib
    digest = hashlib.sha256(t.tobytes()).hexdigest()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, job_ms, bench.weak_value(world, 1000, 4, job_ms), digest))


def test_two_ranks_weak_scaling_and_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]  # both see the slowest rank's time
    assert out[0][2] == pytest.approx(2 * 1000 * 4 / 0.015)  # all ranks' work over the job time
    assert out[0][3] != out[1][3]  # each rank its own domain


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import argparse

    import bench
    args = argparse.Namespace(gpus=2, steps=1, warmup=0)
    assert bench.run_reference(args, rank=1) == 0
    assert capsys.readouterr().out == ""


def _place_rank(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import numpy as np

    import bench
    rng = np.random.default_rng(5)
    fp = [int(x) for x in rng.integers(1, 1000, size=37)]  # the units' footprints, the same on every rank
    mine = bench.place_by_footprint(fp, world)[rank]
    every = bench.gather_over_ranks(mine, world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, fp, every))


def test_units_placed_on_ranks_by_footprint():
    """Ensemble members and served requests go to ranks by device footprint: every rank computes the same
    placement, each unit lands on exactly one rank, and the ranks' loads differ by at most one unit's footprint."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_place_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fp, every0 = out[0][1], out[0][2]
    assert out[1][2] == every0  # the same placement on both ranks
    units = sorted(u for part in every0 for u in part)
    assert units == list(range(len(fp)))
    loads = [sum(fp[u] for u in part) for part in every0]
    assert max(loads) - min(loads) <= max(fp)
