# SPDX-License-Identifier: GPL-3.0-or-later
"""Builds libcw_dycore.so in-tree (cppwrf_b200/lib/) with nvcc for sm_100a.

The FP64 form must round every operation as the reference's CPU build does: --fmad=false (no FMA
contraction), IEEE division and square root (nvcc's defaults: no fast-math flag in FLAGS), and
-ffp-contract=off for the host compiler. The mixed form's step is a separate translation unit with MIXED_FLAGS.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libcw_dycore.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++20", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
         "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr"]
SOURCES = ["cw_runtime.cu", "cw_step_mixed.cu", "cw_case.cpp", "cw_serve.cpp", "cw_output.cpp"]
# The mixed form's kernels (their own translation unit) are held to a tolerance, not to bit identity: FMA
# contraction and single-precision denormals flushed; division and square root stay IEEE (approximate FP32
# division raised the 1 h relative-L2 error of v, phi' and mu' above 1e-4 on the 400 x 400 x 60 case).
MIXED_FLAGS = [f for f in FLAGS if f != "--fmad=false"] + ["--fmad=true", "-ftz=true"]


def build(verbose=False):
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    objs, procs = [], []
    for src in SOURCES:  # the translation units compile in parallel
        obj = os.path.join(HERE, "lib", os.path.splitext(src)[0] + ".o")
        flags = MIXED_FLAGS if src == "cw_step_mixed.cu" else FLAGS
        cmd = [NVCC] + ARCH + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd = [CXX, "-std=c++20", "-O3", "-fPIC", "-ffp-contract=off", "-fopenmp", "-c", os.path.join(CSRC, src),
                   "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-Xcompiler", "-fopenmp", "-lgomp", "-ldl"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
