"""Generate the golden fixtures under tests/golden/ from the reference's own tests.

Run in a container where the reference checkout exists (default path below, or ``--reference``).
The GPU box never runs this script; it only reads the JSON files this script writes.

Sources (paths relative to the reference repository root):
  tests/test_permutation.cpp:20-102   permutation known answers (counts, first/last ranks)
  tests/assets/case1.structure.json   32-site random cell: distance matrix + shell matrix (pymatgen)
  tests/assets/case1.supercell.json   supercell fixture (3x2x1)
  tests/test_structure.cpp:209-238    fcc 3x3x3 naive radii and coordination numbers 12/6/24/12/12/8
  python/tests/test_core.py:28-44     the 16-site systematic settings used by the pytest suite
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_permutation_kats(src: str) -> dict:
    confs = {}
    for name, body in re.findall(r"configuration_t\s+(\w+)\{([^}]*)\};", src):
        vals = [int(v) for v in body.replace("\n", " ").split(",") if v.strip()]
        confs[name] = vals
    counts = {}
    for name, value in re.findall(r"ASSERT_EQ\(num_permutations\((\w+)\),\s*(?:rank_t\{)?(\d+)\}?\)", src):
        counts[name] = int(value)
    first = re.search(r"first_permutations\{([^}]*)\}", src).group(1)
    last = re.search(r"last_permutations\{([^}]*)\}", src).group(1)
    return {
        "configurations": confs,
        "num_permutations": counts,
        "first_permutations": [n.strip() for n in first.split(",") if n.strip()],
        "last_permutations": [n.strip() for n in last.split(",") if n.strip()],
        "all_ranks_case": "conf_first_16",
    }


def parse_structure_kats(src: str) -> dict:
    block = src[src.index("TEST(Structure, prefactors_single)"):]
    dists = re.search(r"assert_vector_is_close\(\s*dists,\s*\{(.*?)\}\);", block, re.S).group(1)
    vals = []
    for tok in dists.replace("\n", " ").split(","):
        tok = tok.strip()
        m = re.fullmatch(r"std::sqrt\(([\d.]+)\)", tok)
        if m:
            vals.append(math.sqrt(float(m.group(1))))
        elif tok.startswith("1.0 / std::sqrt("):
            vals.append(1.0 / math.sqrt(float(tok[len("1.0 / std::sqrt("):-1])))
        else:
            vals.append(float(tok))
    coord = re.search(r"\{(12, 6, 24, 12, 12, 8)\}", block).group(1)
    return {
        "fcc_one_species": {
            "lattice": [[1, 0, 0], [0, 1, 0], [0, 0, 1]],
            "coords": [[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]],
            "species": [1, 1, 1, 1],
            "supercell": [3, 3, 3],
            "naive_distances": vals,
            # distances_naive is called with its own defaults (atol = machine epsilon, rtol = 1e-9,
            # core/structure.h:195-197); the test compares with assert_vector_is_close defaults.
            "naive_rtol": 1.0e-9,
            "compare_atol": 1.0e-5,
            "compare_rtol": 1.0e-3,
            "shell_weights": {str(k): 1 for k in range(1, 7)},
            "coordination_numbers": [int(x) for x in coord.split(",")],
        }
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="root of a dgehringer/sqsgenerator 0.5.6 checkout (its tests/ folder is read)")
    args = ap.parse_args()
    ref = args.reference
    with open(os.path.join(ref, "tests/test_permutation.cpp")) as f:
        perm = parse_permutation_kats(f.read())
    with open(os.path.join(HERE, "permutation_kats.json"), "w") as f:
        json.dump(perm, f, indent=1)
    with open(os.path.join(ref, "tests/test_structure.cpp")) as f:
        st = parse_structure_kats(f.read())
    with open(os.path.join(HERE, "structure_kats.json"), "w") as f:
        json.dump(st, f, indent=1)
    with open(os.path.join(ref, "tests/assets/case1.structure.json")) as f:
        case1 = json.load(f)
    with open(os.path.join(HERE, "case1_structure.json"), "w") as f:
        json.dump(case1, f, separators=(",", ":"))
    with open(os.path.join(ref, "tests/assets/case1.supercell.json")) as f:
        sc = json.load(f)
    with open(os.path.join(HERE, "case1_supercell.json"), "w") as f:
        json.dump(sc, f, separators=(",", ":"))
    print("wrote", sorted(p for p in os.listdir(HERE) if p.endswith(".json")))


if __name__ == "__main__":
    main()
