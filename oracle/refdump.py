# SPDX-License-Identifier: GPL-3.0-or-later
"""TEST INFRASTRUCTURE ONLY: runs the reference's own compiled dycore (oracle/_ref/ref_harness*, built from
the CPPWRF sources by oracle/Makefile) on a capi.Case and returns every field, or times its step loop.
Used by tests/ (parity pins) and by bench.py's CPU-baseline leg (the reference arm)."""
import ctypes as C
import os
import struct
import subprocess
import tempfile

import numpy as np

from cppwrf_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
# a CPPWRF checkout: CPPWRF_REFERENCE, else the directory `reference` beside this repository
REFERENCE_SRC = os.environ.get("CPPWRF_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def available():
    return os.path.isdir(os.path.join(REFERENCE_SRC, "src", "dyn")) or os.path.exists(os.path.join(REF_DIR, "ref_harness"))


def build():
    if not os.path.exists(os.path.join(REF_DIR, "ref_harness_own")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REFERENCE_SRC}"], check=True)


def _vertical_arrays(case):
    v = case.vertical()
    nz = case.g.nz
    arrs = []
    for name in ("znu", "dnw", "rdnw", "c1h", "c2h", "c3h", "c4h"):
        arrs.append(np.ctypeslib.as_array(getattr(v, name), shape=(nz,)))
    for name in ("znw", "dn", "rdn", "fnm", "fnp", "c1f", "c2f", "c3f", "c4f"):
        arrs.append(np.ctypeslib.as_array(getattr(v, name), shape=(nz + 1,)))
    for name in ("u_base", "v_base", "t_base", "qv_base_1d", "z_base"):
        arrs.append(np.ctypeslib.as_array(getattr(v, name), shape=(nz,)))
    scal = [v.cf1, v.cf2, v.cf3, v.cfn, v.cfn1, v.rdx, v.rdy, v.p_top, v.t0]
    return arrs, scal


def write_input(case, nsteps, fin):
    """The harness's input file for case and nsteps."""
    names = [n for n in capi.FIELDS if not n.startswith("Q_")]
    if True:
        with open(fin, "wb") as f:
            f.write(bytes(case.g))
            f.write(bytes(case.o))
            arrs, scal = _vertical_arrays(case)
            for a in arrs:
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
            f.write(struct.pack("<9d", *scal))
            names = [n for n in capi.FIELDS if not n.startswith("Q_")]
            for name in names:
                a, L = case.field(name)
                f.write(struct.pack("<q", a.size))
                f.write(a.astype("<f8").tobytes())
            for n in range(case.o.n_scalars):
                for name in ("Q_1", "Q_2", "Q_TENDF"):
                    a, L = case.field(name, n)
                    f.write(struct.pack("<q", a.size))
                    f.write(a.astype("<f8").tobytes())
            if case.o.lbc:
                for var in range(5):
                    for side in range(4):
                        vals, tends = case.lbc(var, side)
                        f.write(struct.pack("<q", vals.size))
                        f.write(vals.astype("<f8").tobytes())
                        f.write(tends.astype("<f8").tobytes())
                for n in range(case.o.n_scalars):
                    for side in range(4):
                        r = case.lbc(n, side, scalar=True)
                        if r is None:
                            f.write(struct.pack("<q", 0))
                            continue
                        f.write(struct.pack("<q", r[0].size))
                        f.write(r[0].astype("<f8").tobytes())
                        f.write(r[1].astype("<f8").tobytes())
                f.write(struct.pack("<d", case.lbc_time()))
            f.write(struct.pack("<i", nsteps))


def time_steps(case, nsteps, threads=None, own_pow=False):
    """Wall seconds of the reference's step loop (its own CPU FP64 build, OpenMP threads) for nsteps."""
    build()
    exe = os.path.join(REF_DIR, "ref_harness_own" if own_pow else "ref_harness")
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    env.setdefault("OMP_WAIT_POLICY", "passive")
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(case, nsteps, fin)
        r = subprocess.run([exe, fin, fout, "--time"], check=True, capture_output=True, text=True, env=env)
        for line in r.stdout.splitlines():
            if line.startswith("STEP_SECONDS"):
                return float(line.split()[1])
    raise RuntimeError("ref_harness printed no STEP_SECONDS")


def lam_args(w, seed, nsteps):
    """ref_harness --lam arguments of a limited-area case of shape w (nx ny nz dx dt time_step_sound n_moist p_top
    hybrid_opt etac) made by the repository's seeded generator inside the harness, and nsteps."""
    return ["--lam", str(w["nx"]), str(w["ny"]), str(w["nz"]), repr(float(w["dx"])), repr(float(w["dt"])),
            str(w["time_step_sound"]), str(w["n_moist"]), repr(float(w["p_top"])), str(w["hybrid_opt"]),
            repr(float(w["etac"])), str(int(seed)), str(int(nsteps))]


def time_lam(w, seed, nsteps, threads=None):
    """Wall seconds of the reference's step loop (the unmodified build, glibc's math) on a limited-area case
    generated inside the harness: no Python-side input and no library of this repository in the calling process."""
    exe = os.path.join(REF_DIR, "ref_harness")
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    env.setdefault("OMP_WAIT_POLICY", "passive")
    r = subprocess.run([exe] + lam_args(w, seed, nsteps) + ["--time"], check=True, capture_output=True, text=True,
                       env=env)
    for line in r.stdout.splitlines():
        if line.startswith("STEP_SECONDS"):
            return float(line.split()[1])
    raise RuntimeError("ref_harness printed no STEP_SECONDS")


def _read_output(fout, n_scalars):
    names = [n for n in capi.FIELDS if not n.startswith("Q_")]
    out = {}
    with open(fout, "rb") as f:
        for name in names:
            (n,) = struct.unpack("<q", f.read(8))
            out[name] = np.frombuffer(f.read(8 * n), dtype="<f8").copy()
        for q in range(n_scalars):
            for name in ("Q_1", "Q_2", "Q_TENDF"):
                (n,) = struct.unpack("<q", f.read(8))
                out[f"{name}:{q}"] = np.frombuffer(f.read(8 * n), dtype="<f8").copy()
    return out


def run_lam(w, seed, nsteps):
    """{field name: whole allocation} of the reference (the unmodified build) after nsteps on the case
    ref_harness --lam generates."""
    build()
    exe = os.path.join(REF_DIR, "ref_harness")
    with tempfile.TemporaryDirectory() as td:
        fout = os.path.join(td, "out.bin")
        subprocess.run([exe] + lam_args(w, seed, nsteps) + [fout], check=True)
        return _read_output(fout, int(w["n_moist"]))


def run(case, nsteps, own_pow=True, harness=None):
    """{field name: whole allocation} of the reference after nsteps (Q_* keyed 'Q_2:n'); harness: another build of
    the driver (ref_harness_facade: the step replaced by the repository's drop-in)."""
    build()
    exe = os.path.join(REF_DIR, harness or ("ref_harness_own" if own_pow else "ref_harness"))
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(case, nsteps, fin)
        subprocess.run([exe, fin, fout], check=True)
        return _read_output(fout, case.o.n_scalars)
