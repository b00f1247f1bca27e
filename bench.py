# SPDX-License-Identifier: GPL-3.0-or-later
"""Benchmark of the B200 RK3 dynamical core: grid-point-steps/s of the 3-D limited-area workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed] [--impl ours|reference]

Workload (one domain per GPU rank, weak scaling): 119 x 89 x 44 mass points, dx = dy = 15 km, dt = 90 s,
4 acoustic substeps, hybrid sigma-pressure coordinate (etac 0.2), model top 50 hPa, seeded terrain
(1.5 km hill + k^-3 orography up to 800 m), 5 moist species (qv qc qr qi qs) advected positive-definite
at rk 3, specified lateral boundaries (5 rows, relaxation toward the initial state). Every input is
synthetic (cw_gen_lam, seeded). The step's working set (~110 fields of 5.4 MB) is far larger than the
126 MB L2, so no flush is needed between steps.

One JSON line on rank 0: value = all ranks' grid points x steps / max over ranks of the device time of the
K timed steps (CUDA events on the handle's stream), e2e = the same through the C ABI with the prognostic
state (every point of each field's window: domain and halo) copied from / to pinned host memory every step, roofline of the dominant kernel (per-kernel CUDA
events, algorithmic bytes below), and the reference CPU build timed on this host.
"""
import argparse
import ctypes as C
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(nx=119, ny=89, nz=44, dx=15000.0, dt=90.0, time_step_sound=4, p_top=5000.0, n_moist=5,
                hybrid_opt=2, etac=0.2)
METRIC = "RK3 grid-point-steps/s (FP64-exact vs mixed, batched); served p50/p99 latency"
UNIT = "grid-point-steps/s"
# the state a step reads and writes that persists between steps (the e2e copies, per step, both ways)
PROGNOSTIC = ["U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL"]


def make_case(capi, precision, seed=1, w=None, **lam):
    """A limited-area case of the workload's shape (or of w: nx, ny, nz, dx, dt, time_step_sound, ...)."""
    w = dict(WORKLOAD, **(w or {}))
    g = capi.grid(w["nx"], w["ny"], w["nz"], w["dx"], w["dt"], 0.0, dy=w["dx"], p_top=w["p_top"],
                  bc_x=capi.SPECIFIED, bc_y=capi.SPECIFIED)
    o = capi.default_options(None, flat=0, n_moist=w["n_moist"], n_scalars=w["n_moist"], lbc=1,
                             time_step_sound=w["time_step_sound"], precision=precision)
    return capi.Case(g, o).gen_lam(seed=seed, hybrid_opt=w["hybrid_opt"], etac=w["etac"], **lam)


# Algorithmic bytes per mass point of one launch: the distinct 3-D arrays the kernel must read and write,
# each once (staggered extents counted as mass points), for the workload's options (terrain: 3-D base
# fields; 5 moist species; specified boundaries: the held tendencies are read).
ALG_ARRAYS = {
    "k_ls_prep": 7 + 5 + 9,   # u2 v2 w2 al ph2 alb phb + 5 q | ru rv rw alt php ww cqu cqv cqw
    "k_tend": 24 + 5,         # u2 v2 w2 t2 ph2 ru rv rw ww p al alt php pb phb 5 tendf cqu cqv cqw hd | 5 tend
    "k_ss_prep": 15 + 18,     # u2 v2 w2 t2 ph2 u1 v1 w1 t1 ph1 ww p alt pb cqw | 5 state 5 saves ww1 c2a al p pm1 a alpha gamma
    "k_uv": 12 + 2,           # u2 v2 ru_tend rv_tend p al alt ph2 php pb cqu cqv | u2 v2
    "k_ac": 24 + 11,          # u2 v2 u_save v_save ww1 ww_m ru_m rv_m t2 t_save t_tend w2 ph2 rw_tend ph_tend
                              # ph_save phb c2a alt a alpha gamma cqw pm1 | ww ww_m ru_m rv_m t2 t_2save w2 ph2 al p pm1
    "k_finish": 15 + 8,       # u2 v2 w2 t2 ph2 ww 5 saves ww1 hd alb pb | u2 v2 w2 t2 ph2 ww al p
    "k_q_update": 3 + 3 + 1,  # per species: q2 q1 qtf + ru_m rv_m ww_m | qn (one thread updates every species: the
                              # fluxes ru_m rv_m ww_m once, below)
    "k_q_march": 3 + 3 + 1,   # the same update with the species' planes staged by TMA (3-D domains)
    "k_q_update_pd": 4 + 3 + 1,
    "k_q_scale_pd": 2 + 3 + 1,
}


# ---------------------------------------------------------------- multi-GPU plumbing (one domain per rank)
def shard_seed(rank):
    """Each rank advances its own domain of the workload (independent members: weak scaling, no exchange)."""
    return 1 + rank


def place_by_footprint(footprints, world):
    """Independent units (ensemble members, served requests) onto ranks by device footprint: each unit, largest
    first, to the rank holding the fewest bytes so far (ties: the lower rank). The same on every rank (deterministic),
    each unit on exactly one rank. Returns the unit indices of each rank, in unit order."""
    load = [0] * world
    ranks = [[] for _ in range(world)]
    for u in sorted(range(len(footprints)), key=lambda u: (-footprints[u], u)):
        r = min(range(world), key=lambda r: (load[r], r))
        load[r] += footprints[u]
        ranks[r].append(u)
    return [sorted(x) for x in ranks]


def footprint_of(capi, case):
    b = C.c_size_t()
    if capi.load().cw_footprint(C.byref(case.g), C.byref(case.o), C.byref(b)) != 0:
        raise RuntimeError("cw_footprint failed")
    return b.value


def gather_over_ranks(obj, world):
    """Every rank's object on every rank (rank order)."""
    if world <= 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out


def max_over_ranks(value, world, device):
    """The maximum of a per-rank time over all ranks (the job's time): an all-reduce MAX of one number."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(world, pts, steps, ms):
    """Whole-job grid-point-steps/s: every rank's points x steps over the slowest rank's time."""
    return world * pts * steps / (ms / 1000.0)


def clocks_sampler(device):
    """Samples SM clocks and throttle reasons with nvidia-smi every 200 ms until stopped."""
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                              "-i", str(device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return None
    rows = []

    def rd():
        for line in p.stdout:
            rows.append([x.strip() for x in line.split(",")])

    t = threading.Thread(target=rd, daemon=True)
    t.start()
    return p, rows


def clocks_summary(sampler):
    if sampler is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    p, rows = sampler
    p.terminate()
    try:
        p.wait(timeout=5)
    except subprocess.TimeoutExpired:
        p.kill()
    sm, smax, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for r in rows:
        try:
            sm.append(float(r[1]))
            smax.append(float(r[2]))
        except (ValueError, IndexError):
            continue
        for n, v in zip(names, r[5:9]):
            if v.strip().lower() == "active":
                reasons.add(n)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    for path in (os.path.join(ROOT, "MEASURED_PEAKS.json"),):
        try:
            d = json.load(open(path))
            return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
        except (OSError, KeyError, ValueError):
            pass
    return 6650.0, "fallback 6.65 TB/s"


def ncu_traffic(kernel, workload_tag):
    """DRAM bytes per launch of kernel from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload_tag}.md")
    try:
        for line in open(path):
            m = re.match(r"\s*traffic_bytes_per_launch:\s*([0-9.eE+]+)", line)
            if m:
                return float(m.group(1))
    except OSError:
        pass
    return None


def host_description():
    """The host CPU model and glibc version (the reference's CPU results depend on both)."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        glibc = subprocess.run(["ldd", "--version"], capture_output=True, text=True).stdout.splitlines()[0].strip()
    except (OSError, IndexError):
        glibc = None
    return {"cpu_model": model, "glibc": glibc}


def cpu_baseline(seconds_target=15.0, capi=None):
    """The reference's own CPU FP64 build (oracle/_ref/ref_harness: its sources compiled unmodified, glibc's math)
    on a bounded sample of the workload, all host threads. The case is generated inside the harness process
    (ref_harness --lam, the same seeded generator and bytes as make_case), so this leg loads no library of this
    repository. Falls back to the oracle port (one thread) when the reference build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    pts = WORKLOAD["nx"] * WORKLOAD["ny"] * WORKLOAD["nz"]
    ncores = os.cpu_count() or 1
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if os.path.exists(exe):
        import refdump
        t1 = refdump.time_lam(WORKLOAD, 1, 1, threads=ncores)
        n = max(2, min(200, int(seconds_target / max(t1, 1e-3))))
        t = refdump.time_lam(WORKLOAD, 1, n, threads=ncores)
        return {"value": pts * n / t, "unit": UNIT, "cores": ncores, "kind": "reference", **host_description(),
                "sample": f"{n} RK3 steps of the {WORKLOAD['nx']}x{WORKLOAD['ny']}x{WORKLOAD['nz']} workload (seed 1), "
                          f"reference CPU FP64 build (oracle/_ref/ref_harness, OpenMP {ncores} threads, "
                          "OMP_WAIT_POLICY=passive), step loop only"}
    if capi is None:
        from cppwrf_b200 import capi
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle
    case = make_case(capi, capi.FP64)
    orc = _oracle.Oracle(case)
    t0 = time.perf_counter()
    orc.step(1)
    t1 = time.perf_counter() - t0
    n = max(1, min(50, int(seconds_target / max(t1, 1e-3))))
    t0 = time.perf_counter()
    orc.step(n)
    t = time.perf_counter() - t0
    return {"value": pts * n / t, "unit": UNIT, "cores": 1, "kind": "port", **host_description(),
            "sample": f"{n} RK3 steps of the workload, the oracle (C restatement, 1 thread)"}


def lam_config(precision, world):
    """The `config` of the headline line: the same dict in both arms."""
    return {"workload": f"lam_119x89x44_{precision}", **WORKLOAD, "moist_species": "qv qc qr qi qs (PD at rk 3)",
            "lbc": "specified, width 5", "seed": 1, "parallelism": f"one domain per GPU x{world}",
            "l2": "inputs larger than L2: ~110 fields x 5.4 MB per step, no flush"}


def run_reference(args, rank):
    """The reference arm: the reference's own CPU implementation of the path on this host's cores, for the same
    workload, metric and config as our arm (rank 0 only; other ranks exit without work)."""
    if rank != 0:
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    cb = cpu_baseline(seconds_target=20.0)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (cw_gen_lam, seeded)",
            "config": lam_config("fp64", world), "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line["ms_per_step"] = 1000.0 * WORKLOAD["nx"] * WORKLOAD["ny"] * WORKLOAD["nz"] / cb["value"]
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- further workloads (precision, ensemble, served)
def _timed_steps(torch, stream, fn, steps):
    """device ms of fn(steps) on stream (CUDA events)."""
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _errors(capi, a_dom, b_dom, case):
    """relative L2 and max-abs of the mixed form against the FP64 form per prognostic (interior points)."""
    out = {}
    names = {"u": ("U_2", 0), "v": ("V_2", 0), "w": ("W_2", 0), "theta": ("T_2", 0), "phi'": ("PH_2", 0),
             "mu'": ("MU_2", 0), "qv": ("Q_2", 0)}
    for key, (name, n) in names.items():
        L = b_dom.layout(name, n)
        a = capi.interior(a_dom.field(name, n), L)
        b = capi.interior(b_dom.field(name, n), L)
        d = a - b
        out[key] = {"rel_l2": float(np.linalg.norm(d) / max(np.linalg.norm(b), 1e-300)),
                    "max_abs": float(np.max(np.abs(d))), "finite": bool(np.all(np.isfinite(a)))}
    return out


PRECISION_WORKLOAD = dict(nx=400, ny=400, nz=60, dx=3000.0, dt=18.0, time_step_sound=6)  # make_case seed 3


def run_precision(args, torch, capi, Domain):
    """400 x 400 x 60 at dx 3 km, dt 18 s, 6 acoustic substeps: the mixed form against the FP64 form (which is
    bit-identical to the oracle) at 1 h and 6 h of simulated time, and the throughput of both."""
    w = dict(PRECISION_WORKLOAD)
    lib = capi.load()
    doms, stream = {}, torch.cuda.Stream()
    for prec in (capi.FP64, capi.MIXED):
        c = make_case(capi, prec, seed=3, w=w)
        d = Domain(c.g, c.o).upload_case(c)
        lib.cw_set_stream(d.h, C.c_void_p(stream.cuda_stream))
        if not args.no_autotune:
            d.set_autotune(True)  # the first steps (ordinary steps, timed with the rest) pick the kernels' shapes
        doms[prec] = d
    pts = w["nx"] * w["ny"] * w["nz"]
    res, times = {}, {capi.FP64: 0.0, capi.MIXED: 0.0}
    done = 0
    for hours in (1, 6):
        target = int(round(hours * 3600 / w["dt"]))
        for prec, d in doms.items():
            times[prec] += _timed_steps(torch, stream, d.step, target - done)
        done = target
        res[f"{hours}h"] = _errors(capi, doms[capi.MIXED], doms[capi.FP64], None)
    v64 = pts * done / (times[capi.FP64] / 1000.0)
    v32 = pts * done / (times[capi.MIXED] / 1000.0)
    line = {"metric": METRIC, "value": v32, "unit": UNIT, "n_gpus": 1, "steps": done, "warmup": 0,
            "ms_per_step": times[capi.MIXED] / done, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (cw_gen_lam, seeded)",
            "config": {"workload": "precision_400x400x60", **w, "n_moist": 5, "hybrid_opt": 2},
            "fp64_value": v64, "mixed_over_fp64": v32 / v64, "errors_mixed_vs_fp64": res}
    print(json.dumps(line), flush=True)
    return 0


def ensemble_members(rng, n=64):
    out = []
    for m in range(n):
        out.append(dict(nx=int(rng.integers(60, 201)), ny=int(rng.integers(60, 201)),
                        nz=int(rng.choice([35, 44, 50, 60])), seed=1000 + m))
    return out


def run_ensemble(args, torch, capi, Domain, Batch, rank=0, world=1):
    """64 members of uneven sizes (nx, ny in [60, 200], nz in {35, 44, 50, 60}, dx 15 km): the batched mixed
    and FP64 forms against the members run one after the other as plain FP64 domains. With several ranks the
    members are placed on the ranks by device footprint (place_by_footprint; no data-path collective) and the job
    time is the slowest rank's (strong scaling: the ensemble is fixed)."""
    lib = capi.load()
    rng = np.random.default_rng(2024)
    spec_all = ensemble_members(rng)
    cases_all = [make_case(capi, capi.FP64, seed=m["seed"], w=m, theta_pert=0.5, wind_pert=1.0) for m in spec_all]
    mine = place_by_footprint([footprint_of(capi, c) for c in cases_all], world)[rank]
    spec = [spec_all[u] for u in mine]
    cases = [cases_all[u] for u in mine]
    stream = torch.cuda.Stream()
    gp_all = sum(m["nx"] * m["ny"] * m["nz"] for m in spec_all)
    out = {}
    for prec in (capi.MIXED, capi.FP64):
        opts = []
        for c in cases:
            o = capi.Options.from_buffer_copy(c.o)
            o.precision = prec
            opts.append(o)
        b = Batch([c.g for c in cases], opts)
        for k, c in enumerate(cases):
            b.upload_case(k, c)
        lib.cw_set_stream(b.h, C.c_void_p(stream.cuda_stream))
        if not args.no_autotune:
            b.set_autotune(True)  # the warm-up steps pick the batch's block shapes and warps per column block
        b.step(args.warmup)
        if world > 1:
            torch.distributed.barrier()
        ms = max_over_ranks(_timed_steps(torch, stream, b.step, args.steps), world, "cuda")
        out[prec] = (gp_all * args.steps / (ms / 1000.0), ms / args.steps, b.launches() // max(args.steps, 1))
        b.close()
    # plain FP64: every member alone, one after the other (each rank its own members), each tuned for itself
    plain_ms = 0.0
    for c in cases:
        d = Domain(c.g, c.o).upload_case(c)
        lib.cw_set_stream(d.h, C.c_void_p(stream.cuda_stream))
        if not args.no_autotune:
            d.set_autotune(True)
            d.step(args.warmup)
        else:
            d.step(1)
        plain_ms += _timed_steps(torch, stream, d.step, args.steps)
        d.close()
    plain_ms = max_over_ranks(plain_ms, world, "cuda")
    plain = gp_all * args.steps / (plain_ms / 1000.0)
    line = {"metric": METRIC, "value": out[capi.MIXED][0], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out[capi.MIXED][1], "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (cw_gen_lam, seeded; per-member theta and wind noise)",
            "config": {"workload": "ensemble_64", "members": len(spec_all), "grid_points": gp_all, "dx": 15000.0,
                       "dt": 90.0, "time_step_sound": 4, "sizes_seed": 2024,
                       "placement": f"members on {world} rank(s) by device footprint"},
            "members_per_rank": [len(x) for x in gather_over_ranks(mine, world)],
            "fp64_batched_value": out[capi.FP64][0], "fp64_plain_serial_value": plain,
            "mixed_batched_over_fp64_plain": out[capi.MIXED][0] / plain,
            "launches_per_step": out[capi.MIXED][2]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def served_requests(rng, n, rate):
    t, out = 0.0, []
    for r in range(n):
        t += float(rng.exponential(1.0 / rate))
        nx = int(round(np.exp(rng.uniform(np.log(40), np.log(300)))))
        ny = int(round(np.exp(rng.uniform(np.log(40), np.log(300)))))
        out.append(dict(t=t, nx=nx, ny=ny, nz=int(rng.integers(35, 61)), steps=int(rng.integers(30, 361)),
                        seed=5000 + r))
    return out


def run_served(args, torch, capi, Domain, Server, rank=0, world=1):
    """Poisson arrivals of forecast requests (40..300 squared, nz 35..60, 30..360 steps) into the served
    mixed-precision form under a 150 GB budget: p50 / p99 latency and aggregate gp-steps/s, beside the same
    requests solved one after the other as plain FP64 domains. With several ranks each request goes to a rank by
    device footprint (place_by_footprint over the stream; each rank serves its requests at their arrival times)."""
    lib = capi.load()
    rng = np.random.default_rng(77)
    reqs_all = served_requests(rng, args.requests, args.rate)
    cases_all = [make_case(capi, capi.MIXED, seed=r["seed"], w=r) for r in reqs_all]
    mine = place_by_footprint([footprint_of(capi, c) for c in cases_all], world)[rank]
    reqs = [reqs_all[u] for u in mine]
    cases = [cases_all[u] for u in mine]
    srv = Server(budget_bytes=150e9, precision=capi.MIXED, keep_results=False)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for r, c in zip(reqs, cases):
        dt = r["t"] - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        srv.submit(c, r["steps"])
    srv.drain()
    st = srv.stats()
    lat = []
    for rid in srv.cases:
        try:
            lat.append(srv.latency(rid))
        except Exception:  # noqa: BLE001 - a failed request has no latency (counted in served_stats)
            pass
    wall = time.perf_counter() - t0
    srv.close()
    gps = sum(r["nx"] * r["ny"] * r["nz"] * r["steps"] for r in reqs)
    if world > 1:  # the job: every rank's requests over the slowest rank's wall time, latencies of all requests
        lat = [x for part in gather_over_ranks(lat, world) for x in part]
        wall_job = max(gather_over_ranks(wall, world))
        st = dict(st, p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
                  mean_s=float(np.mean(lat)), gp_steps_per_s=sum(gather_over_ranks(gps, world)) / wall_job)
    # plain FP64, one request after the other: the device time of the steps alone, and the wall time of the
    # whole solve (domain set-up, upload, steps, read-back of the prognostic state), the served path's equal
    stream = torch.cuda.Stream()
    plain_ms, plain_wall = 0.0, 0.0
    for r in reqs:
        c = make_case(capi, capi.FP64, seed=r["seed"], w=r)
        t0 = time.perf_counter()
        d = Domain(c.g, c.o).upload_case(c)
        lib.cw_set_stream(d.h, C.c_void_p(stream.cuda_stream))
        plain_ms += _timed_steps(torch, stream, d.step, r["steps"])
        for name in ("U_2", "V_2", "W_2", "T_2", "PH_2", "MU_2", "P", "AL"):
            d.field(name)
        d.close()
        plain_wall += time.perf_counter() - t0
    gps_job = sum(gather_over_ranks(gps, world))
    plain = gps_job / (max_over_ranks(plain_ms, world, "cuda") / 1000.0)
    plain_w = gps_job / max(gather_over_ranks(plain_wall, world))
    line = {"metric": METRIC, "value": st["gp_steps_per_s"], "unit": UNIT, "n_gpus": world, "steps": None,
            "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic (cw_gen_lam, seeded per request; Poisson arrivals)",
            "config": {"workload": "served_stream", "requests": len(reqs), "rate_per_s": args.rate,
                       "hbm_budget_bytes": 150e9, "sizes": "log-uniform 40..300, nz 35..60, 30..360 steps"},
            "p50_latency_s": st["p50_s"], "p99_latency_s": st["p99_s"], "mean_latency_s": st["mean_s"],
            "served_stats": st, "fp64_plain_serial_value": plain, "served_over_fp64_plain": st["gp_steps_per_s"] / plain,
            "fp64_plain_serial_wall_value": plain_w, "served_over_fp64_plain_wall": st["gp_steps_per_s"] / plain_w,
            "note": "value = completed gp-steps / (last completion - first submission), host clock, arrival gaps "
                    "included; fp64_plain_serial_value: device time of the steps only; _wall_value: whole solves"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default block shapes")
    ap.add_argument("--workload", choices=["lam", "precision", "ensemble", "served"], default="lam",
                    help="lam: the headline 119x89x44 line; precision: 400x400x60 mixed vs FP64 with 1 h / 6 h errors; "
                         "ensemble: 64 uneven members; served: Poisson requests under an HBM budget (members and "
                         "requests placed on the ranks by device footprint when N > 1)")
    ap.add_argument("--requests", type=int, default=24, help="served: number of requests")
    ap.add_argument("--rate", type=float, default=2.0, help="served: Poisson arrival rate per second")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if not args.no_autotune:
        args.warmup = max(args.warmup, 8)  # 6 tuning steps, the graph capture, one replay
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    import torch.distributed as dist

    from cppwrf_b200 import Domain, capi

    torch.cuda.set_device(local)
    if args.workload != "lam":
        from cppwrf_b200 import Batch, Server
        capi.load().cw_use_device(local)
        if args.workload == "precision":  # one domain pair: rank 0 alone
            return run_precision(args, torch, capi, Domain) if rank == 0 else 0
        if world > 1:  # ensemble members / served requests placed on the ranks by footprint
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            import datetime
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        try:
            if args.workload == "ensemble":
                return run_ensemble(args, torch, capi, Domain, Batch, rank, world)
            return run_served(args, torch, capi, Domain, Server, rank, world)
        finally:
            if world > 1:
                dist.destroy_process_group()
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    lib = capi.load()
    lib.cw_use_device(local)
    prec = capi.MIXED if args.precision == "mixed" else capi.FP64
    case = make_case(capi, prec, seed=shard_seed(rank))
    dom = Domain(case.g, case.o).upload_case(case)
    if not args.no_autotune:
        dom.set_autotune(True)  # the first warm-up steps pick each point kernel's block shape
    stream = torch.cuda.Stream()  # a dedicated stream: the handle launches on it, the events are recorded on it
    lib.cw_set_stream(dom.h, C.c_void_p(stream.cuda_stream))
    pts = WORKLOAD["nx"] * WORKLOAD["ny"] * WORKLOAD["nz"]

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up (the first step captures the CUDA graph)
    dom.step(args.warmup)
    torch.cuda.synchronize()
    sampler = clocks_sampler(local)
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dom.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = clocks_summary(sampler)
    ms = e0.elapsed_time(e1)
    launches = dom.launches()
    ms = max_over_ranks(ms, world, "cuda")
    value = weak_value(world, pts, args.steps, ms)

    # e2e: the prognostic state from pinned host memory, one step, the state back, every step
    host = {}
    for name in PROGNOSTIC:
        L = dom.layout(name)
        host[name] = torch.empty(L.total, dtype=torch.float64).pin_memory()
        host[name].copy_(torch.from_numpy(dom.field(name)))
    qhost = []
    for n in range(case.o.n_scalars):
        L = dom.layout("Q_2", n)
        t = torch.empty(L.total, dtype=torch.float64).pin_memory()
        t.copy_(torch.from_numpy(dom.field("Q_2", n)))
        qhost.append(t)
    # the window points of each field (domain and halo; the allocations' row padding is not copied)
    def window_points(L):
        if L.uniform:
            return L.total
        return (L.wi1 - L.wi0) * (L.wj1 - L.wj0) * (L.nz if L.rank == 3 else 1)
    ebytes = sum(window_points(dom.layout(n)) * 8 for n in host) + \
        sum(window_points(dom.layout("Q_2", q)) * 8 for q in range(len(qhost)))
    dp = C.POINTER(C.c_double)
    n_e2e = max(3, min(args.steps, 20))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    # every field of the state in one cw_upload_windows / cw_download_windows call (one synchronisation per step)
    tensors = list(host.values()) + qhost
    nf = len(tensors)
    fids = (C.c_int * nf)(*([capi.F[name] for name in host] + [capi.F["Q_2"]] * len(qhost)))
    fns = (C.c_int * nf)(*([0] * len(host) + list(range(len(qhost)))))
    fptr = (dp * nf)(*[C.cast(t.data_ptr(), dp) for t in tensors])
    fcnt = (C.c_size_t * nf)(*[t.numel() for t in tensors])
    for _ in range(n_e2e):
        lib.cw_upload_windows(dom.h, 0, nf, fids, fns, fptr, fcnt)
        lib.cw_step(dom.h, 1)
        lib.cw_download_windows(dom.h, 0, nf, fids, fns, fptr, fcnt)
    g1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ems = max(g0.elapsed_time(g1), wall * 1000.0)
    ems = max_over_ranks(ems, world, "cuda")
    e2e = weak_value(world, pts, n_e2e, ems)

    # per-kernel device time (eager steps with events around each launch); dominant kernel's roofline
    nk = C.c_int()
    lib.cw_profile(dom.h, 2, C.byref(nk))
    table = []
    for k in range(nk.value):
        nm = C.create_string_buffer(64)
        kms, kn = C.c_double(), C.c_longlong()
        lib.cw_profile_entry(dom.h, k, nm, 64, C.byref(kms), C.byref(kn))
        table.append((nm.value.decode(), kms.value, kn.value))
    table.sort(key=lambda r: -r[1])
    total_ms = sum(r[1] for r in table)
    dom_name, dom_ms, dom_n = next((r for r in table if r[0] in ALG_ARRAYS), table[0])
    esz = 4 if prec == capi.MIXED else 8
    arrays = ALG_ARRAYS.get(dom_name, 0) * (WORKLOAD["n_moist"] if dom_name.startswith("k_q_") else 1)
    if dom_name in ("k_q_update", "k_q_march"):
        arrays = 4 * WORKLOAD["n_moist"] + 3
    alg_bytes = arrays * pts * esz
    avg_s = dom_ms / 1000.0 / dom_n
    peak, peak_src = measured_peak()
    achieved = alg_bytes / avg_s / 1e9
    tag = f"lam119x89x44_{args.precision}"
    traffic = ncu_traffic(dom_name, tag)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": f"the committed ncu summary profiles/{dom_name}_{tag}.md (not measured in "
                                                     "this run)" if traffic is not None else None,
                "kernel": dom_name, "algorithmic_bytes_per_launch": alg_bytes,
                "avg_launch_ms": dom_ms / dom_n, "peak_source": peak_src,
                "kernel_share": {r[0]: round(r[1] / total_ms, 4) for r in table[:8]}}
    # the whole step against the per-grid-point traffic model (4 416 B FP64 / 2 208 B FP32 per point-step)
    step_bytes = 4416 if prec == capi.FP64 else 2208
    step_roofline = {"bytes_per_gp_step": step_bytes, "achieved_GBps": value / world * step_bytes / 1e9,
                     "frac": value / world * step_bytes / 1e9 / peak}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == capi.FP64 else "f32+f64",
            "data": "synthetic (cw_gen_lam, seeded)",
            "config": lam_config(args.precision, world),
            "block_shapes": {k: ["128x1", "64x2", "32x4"][dom.autotune_choice(k)]
                             for k in ("k_tend", "k_tend_b", "k_tendf_rk1", "k_uv", "k_q_update", "k_q_face_pd",
                                       "k_q_scale_pd", "k_q_update_pd", "k_p_rho_phi")
                             if dom.autotune_choice(k) >= 0},
            "level_chunks": {k: [2, 1, 4][dom.autotune_choice(k)] for k in ("k_q_march",) if dom.autotune_choice(k) >= 0},
            "column_warps": {k: [8, 16, 4][dom.autotune_choice(k)]
                             for k in ("k_ls_prep", "k_ss_prep", "k_ac", "k_finish") if dom.autotune_choice(k) >= 0},
            "clocks": clocks, "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": ebytes,
                                      "d2h_bytes_per_step": ebytes, "steps": n_e2e},
            "gpu_launches": launches, "roofline": roofline, "step_roofline": step_roofline}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(capi=capi)
        except Exception as e:  # noqa: BLE001 - reported, not fatal
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    dom.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
