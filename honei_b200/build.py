"""Builds libhonei_b200.so in-tree for sm_100a with nvcc (no torch extension machinery).

    python -m honei_b200.build          # incremental: rebuilds objects whose sources changed

The library is plain CUDA C++ behind the C ABI in include/honei_b200.h.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhonei_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false is not needed: every rounding-sensitive operation uses the _rn intrinsics.
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I" + os.path.join(ROOT, "include")]


def _deps():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h")))


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    dep_mtime = max([os.path.getmtime(d) for d in _deps()] + [0])
    objs = []
    procs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if (not ptxas_info and os.path.exists(o) and os.path.getmtime(o) >= os.path.getmtime(s)
                and os.path.getmtime(o) >= dep_mtime):
            continue
        cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
        if s.endswith(".cpp"):
            cmd = [NVCC] + FLAGS + ["-x", "cu"] + ARCH + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd))
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for s, p in procs:
        out = p.communicate()[0].decode()
        if out.strip() and (verbose or ptxas_info or p.returncode):
            print(out)
        if p.returncode:
            failed.append(s)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    if (not os.path.exists(LIB) or procs
            or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcuda"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
