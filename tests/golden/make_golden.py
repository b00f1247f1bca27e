# SPDX-License-Identifier: GPL-3.0-or-later
"""Extracts the reference's FP64 regression goldens into tests/golden/reference_snapshots.json.

CPPWRF ships, for each ideal case, the end state of its CPU FP64 build after two steps
(tools/regression/golden/<case>_cpu_fp64/snap_000002.{json,bin}, runs made by
tools/regression/run.sh --quick; run lengths at run.sh:146-150) and the run's diag.csv (one row per
step, io::DiagWriter). This script records, per variable of each snapshot, the SHA-256 of its
little-endian float64 bytes in the snapshot's (k, j, i) order plus its shape and a few sample values,
the snapshot's JSON text and the diag.csv lines verbatim, together with the case's configuration
(configs/<case>.ini). The oracle test recomputes the same variables and compares hashes, which is a
bit-for-bit comparison without committing megabytes of binary data.

Run from the repository root, with a CPPWRF checkout named by CPPWRF_REFERENCE (default: the directory
`reference` beside this repository):
    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("CPPWRF_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference")

# configs/<case>.ini of the reference, with the quick-mode run_time of run.sh:146-150
CASES = {
    "straka": dict(kind="straka", nx=512, ny=1, nz=64, dx=100.0, dy=100.0, ztop=6400.0, bc_x="periodic",
                   bc_y="periodic", dt=1.0, khdif=75.0, kvdif=75.0, pr_inv=1.0, run_time=2.0),
    "warm_bubble": dict(kind="warm_bubble", nx=200, ny=1, nz=100, dx=100.0, dy=100.0, ztop=10000.0,
                        bc_x="symmetric", bc_y="periodic", dt=1.0, khdif=0.0, kvdif=0.0, pr_inv=3.0,
                        run_time=2.0),
    "igw": dict(kind="igw", nx=300, ny=1, nz=10, dx=1000.0, dy=1000.0, ztop=10000.0, bc_x="periodic",
                bc_y="periodic", dt=6.0, khdif=0.0, kvdif=0.0, pr_inv=3.0, run_time=12.0),
    "rest_state": dict(kind="rest_state", nx=24, ny=24, nz=40, dx=2000.0, dy=2000.0, ztop=20000.0,
                       bc_x="periodic", bc_y="periodic", dt=10.0, khdif=0.0, kvdif=0.0, pr_inv=3.0,
                       run_time=20.0),
    # moist convection with Kessler microphysics (configs/squall2d.ini: species qv, qc, qr; mp_physics = 1)
    "squall2d": dict(kind="squall2d", nx=120, ny=1, nz=40, dx=1000.0, dy=1000.0, ztop=20000.0, bc_x="periodic",
                     bc_y="periodic", dt=6.0, khdif=0.0, kvdif=0.0, pr_inv=3.0, run_time=12.0, n_moist=3,
                     mp_physics=1),
}


def main():
    out = {"source": "CPPWRF tools/regression/golden/*_cpu_fp64/snap_000002 (golden/COMMIT "
                     + open(os.path.join(REF, "tools/regression/golden/COMMIT")).read().strip() + ")",
           "cases": {}}
    for name, cfg in CASES.items():
        d = os.path.join(REF, "tools/regression/golden", f"{name}_cpu_fp64")
        meta = json.load(open(os.path.join(d, "snap_000002.json")))
        raw = open(os.path.join(d, "snap_000002.bin"), "rb").read()
        vars_ = {}
        for v in meta["variables"]:
            a = np.frombuffer(raw[v["offset"]:v["offset"] + v["nbytes"]], dtype="<f8").reshape(v["shape"])
            vars_[v["name"]] = {
                "shape": v["shape"],
                "sha256": hashlib.sha256(a.astype("<f8").tobytes()).hexdigest(),
                "sum": float(a.sum()),
                "samples": [float(x) for x in a.ravel()[:: max(1, a.size // 7)][:8]],
            }
        snap_json = open(os.path.join(d, "snap_000002.json")).read()
        diag_csv = open(os.path.join(d, "diag.csv")).read().splitlines()
        out["cases"][name] = {"config": cfg, "step": meta["step"], "time": meta["time"], "variables": vars_,
                              "snap_json": snap_json, "diag_csv": diag_csv}
    path = os.path.join(HERE, "reference_snapshots.json")
    json.dump(out, open(path, "w"), indent=1)
    print("wrote", path)


if __name__ == "__main__":
    sys.exit(main())
