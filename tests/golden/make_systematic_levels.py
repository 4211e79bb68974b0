"""Exhaustive oracle enumeration of the fcc 2x2x2 (32-site) A16B16 cell: all C(32,16) = 601,080,390
permutations. Writes the keep+1 best distinct objectives with their exact configuration counts and
rank checksums to tests/golden/fcc32_systematic_levels.json.

The workload is the systematic configuration of the benchmark: a = 4.0 A, shells 1 and 2 with weights
1.0 / 0.5, all pair weights 1, target 0, keep 10, prefactors computed. Geometry comes from the oracle's
own restatement (oracle/geometry.py), independent of the product's C++ precompute. Takes about a
minute on 8 cores.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from oracle import geometry as G  # noqa: E402


def fcc32_sublattice(T):
    lat, frac = G.fcc(4.0)
    L, F, species = G.supercell(lat, frac, [1] * 4, 2, 2, 2, T)
    comp = [(set(range(32)), {13: 16, 22: 16})]
    dmat = G.distance_matrix(L, F, T)
    radii = G.distances_histogram(dmat, 0.05, 0.25, T)
    weights = {1: T(1.0), 2: T(0.5)}
    K, S = 2, 2
    pw = np.ones((S, K, K), dtype=T)
    return G.prepare_interact(L, F, species, comp, radii, weights, T, pair_weights=pw)


def main():
    out = {"workload": "fcc 2x2x2 A16B16 systematic, shells 1/2 weights 1.0/0.5, pair weights 1, keep 10",
           "num_permutations": 601080390, "keep": 10}
    for prec, T in (("double", np.float64), ("single", np.float32)):
        sd = fcc32_sublattice(T)
        t = time.time()
        lv = oracle.systematic_levels(sd, prec=prec, keep=10)
        out[prec] = [{"objective": v, "count": c, "checksum": s} for v, c, s in lv]
        print(prec, f"{time.time() - t:.1f}s", lv[:2])
    with open(os.path.join(HERE, "fcc32_systematic_levels.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
