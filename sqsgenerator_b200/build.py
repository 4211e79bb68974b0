"""Build the native library ``sqsgenerator_b200/_lib/libsqsg_b200.so`` in-tree with nvcc.

Device code targets sm_100a only. ``--fmad=false`` plus ``-ffp-contract=off`` on the host side keep
every floating-point operation separately rounded, which the bit-exact objective relies on (the
device objective also uses explicit ``__dmul_rn``/``__dadd_rn`` style intrinsics). Every source is
compiled to its own object in parallel (the engine kernels live in separate translation units), then
the objects are linked into one shared library.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libsqsg_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["engine.cu", "kernel_mask.cu", "kernel_wide.cu", "kernel_lat.cu", "kernel_lat2.cu", "kernel_lat5.cu", "kernel_latw.cu", "kernel_materialize.cu", "geometry.cpp", "microbench.cu", "no_alloc.cu",
           "prepare.cu", "select.cu"]
HEADERS = ["attr_tracker.h", "engine.cuh", "engine_device.cuh", "host_copy.h", "kernels.h", "permutation.h", "philox.cuh",
           "prepare.h", "select.h", "sqsg_internal.h", "tiles.h", "tuning_table.inc"]
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "--fmad=false",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-O2"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "sqsgen_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs() if os.path.exists(f))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *FLAGS, "-I", INCLUDE, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    workers = max(1, min(len(SOURCES), os.cpu_count() or 1))
    # the kernel translation units take longest: start them first
    order = sorted(SOURCES, key=lambda f: 0 if f.startswith("kernel_") else 1)
    with cf.ThreadPoolExecutor(workers) as ex:
        objs = dict(zip(order, ex.map(lambda f: _compile(f, verbose), order)))
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *[objs[f] for f in SOURCES],
           "-o", LIB + ".tmp", "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
