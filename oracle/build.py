"""Build recipe for the oracle's C++ restatement (test infrastructure only).

Compiles ``oracle/sqsg_oracle.cpp`` into ``oracle/liboracle.so`` with the flags the restatement
needs for bit-exact scalar arithmetic: no FMA contraction and no fast-math.

The reference itself (``include/sqsgen/**`` of dgehringer/sqsgenerator) is not compiled: it needs
Eigen3, Boost.Multiprecision, Abseil and BS_thread_pool, none of which is installed, so there is no
``oracle/_ref`` build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "sqsg_oracle.cpp")
OUT = os.path.join(HERE, "liboracle.so")

FLAGS = ["-O2", "-std=c++20", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread"]


def build(force: bool = False) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    cmd = ["g++", *FLAGS, SRC, "-o", OUT + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
