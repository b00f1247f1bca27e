# SPDX-License-Identifier: GPL-3.0-or-later
"""Builds libcw_dycore.so in-tree (cppwrf_b200/lib/) with nvcc for sm_100a.

The FP64 form must round every operation as the reference's CPU build does: --fmad=false (no FMA
contraction), IEEE division and square root (nvcc's defaults, asserted below by the absence of any
fast-math flag), and -ffp-contract=off for the host compiler.
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
SOURCES = ["cw_runtime.cu", "cw_case.cpp", "cw_serve.cpp", "cw_output.cpp"]


def build(verbose=False):
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(HERE, "lib", os.path.splitext(src)[0] + ".o")
        cmd = [NVCC] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd = [CXX, "-std=c++20", "-O3", "-fPIC", "-ffp-contract=off", "-fopenmp", "-c", os.path.join(CSRC, src),
                   "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-Xcompiler", "-fopenmp", "-lgomp"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
