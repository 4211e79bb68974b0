"""Build the native library ``sqsgenerator_b200/_lib/libsqsg_b200.so`` in-tree with nvcc.

Device code targets sm_100a only. ``--fmad=false`` plus ``-ffp-contract=off`` on the host side keep
every floating-point operation separately rounded, which the bit-exact objective relies on (the
device objective also uses explicit ``__dmul_rn``/``__dadd_rn`` style intrinsics).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libsqsg_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["engine.cu", "geometry.cpp", "microbench.cu", "no_alloc.cu", "select.cu"]
HEADERS = ["engine.cuh", "engine_device.cuh", "permutation.h", "philox.cuh", "select.h", "sqsg_internal.h",
           "tiles.h"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "sqsgen_b200.h"))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs() if os.path.exists(f))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [
        nvcc(),
        "-O3",
        "-std=c++17",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-lineinfo",
        "--fmad=false",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
        "-shared",
        "-I", INCLUDE,
        *[os.path.join(CSRC, f) for f in SOURCES],
        "-o", LIB + ".tmp",
        "-lcudart",
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
