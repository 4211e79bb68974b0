"""The native library without a GPU: exports, host precompute against the oracle, permutation math,
the reference-schema parser (CPU only; no device compute is called)."""
import json
import os
import re

import numpy as np
import pytest

import cases
import oracle
from oracle import geometry as G
import sqsgenerator_b200 as S
from sqsgenerator_b200 import _native as N
from sqsgenerator_b200.core import ParseErrorCode

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def header_symbols():
    out = set()
    inc = os.path.join(ROOT, "include")
    for name in os.listdir(inc):
        if name.endswith(".h"):
            with open(os.path.join(inc, name)) as f:
                src = f.read()
            out |= set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(sqsg_\w+)\s*\(", src, re.M))
    return out


def test_library_loads_and_exports_header_symbols():
    L = N.lib()
    declared = header_symbols()
    assert "sqsg_optimize" in declared and len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    assert set(N.EXPORTED) <= declared
    assert N.version().startswith("sqsgen_b200")


def test_no_device_is_an_error_not_a_fallback():
    if N.device_count() > 0:
        pytest.skip("a CUDA device is visible")
    with pytest.raises(N.NativeError) as e:
        S.optimize(cases.fcc32(iterations=1000))
    assert e.value.status_name == "SQSG_ERR_CUDA"


# --------------------------------------------------------------------------- host precompute parity
@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_distance_matrix_matches_oracle(T):
    d = json.load(open(os.path.join(GOLDEN, "case1_structure.json")))
    a = N.distance_matrix(d["lattice"], d["frac_coords"], dtype=T)
    b = G.distance_matrix(d["lattice"], d["frac_coords"], T)
    assert np.array_equal(a, b)


def test_shells_and_radii_match_oracle():
    d = json.load(open(os.path.join(GOLDEN, "case1_structure.json")))
    D = N.distance_matrix(d["lattice"], d["frac_coords"])
    eps = np.finfo(np.float64).eps
    r1 = N.distances_naive(D, eps, 1e-9)
    r2 = G.distances_naive(D, eps, 1e-9)
    assert np.array_equal(r1, np.array(r2))
    sm = N.shell_matrix(D, r1, eps, 1e-9)
    assert np.array_equal(sm, np.array(d["shell_matrix"]))


@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_peak_radii_match_oracle(T):
    for cells in ((2, 2, 2), (3, 3, 3)):
        lat, frac = G.fcc(4.0)
        L, F, _ = N.supercell(lat, frac, [1] * 4, *cells, dtype=T)
        D = N.distance_matrix(L, F, dtype=T)
        assert np.array_equal(N.distances_histogram(D, 0.05, 0.25), np.array(G.distances_histogram(D, 0.05, 0.25, T), T))


def test_prefactors_and_pairs_match_oracle():
    k = json.load(open(os.path.join(GOLDEN, "structure_kats.json")))["fcc_one_species"]
    L, F, Sp = N.supercell(k["lattice"], k["coords"], k["species"], *k["supercell"])
    D = N.distance_matrix(L, F)
    eps = np.finfo(np.float64).eps
    radii = N.distances_naive(D, eps, 1e-9)
    sm = N.shell_matrix(D, radii, eps, 1e-9)
    f = N.prefactors(sm, [1, 2, 3, 4, 5, 6], Sp)
    assert G.coordination_numbers(f, len(Sp)) == k["coordination_numbers"]
    w = {s: 1.0 for s in [1, 2, 3]}
    assert np.array_equal(N.pairs(sm, list(w)), G.pairs(sm, w))


def test_sort_by_sublattice_matches_oracle():
    rng = np.random.default_rng(1)
    for n_sl in (1, 2, 3):
        sl_of = rng.integers(0, n_sl + 1, size=40)
        comp = [(set(np.flatnonzero(sl_of == k).tolist()), {1: 1}) for k in range(n_sl)]
        order, windows = N.sort_by_sublattice(sl_of, n_sl)
        o2, b2 = G.shuffling_bounds(40, comp)
        assert [tuple(w) for w in windows.tolist()] == [tuple(b) for b in b2]
        assert order.tolist() == list(o2)


def test_prepare_matches_oracle_precompute():
    """The product's pair list / packed species / prefactors / scaled weights equal the oracle's."""
    c = S.parse_config(cases.fcc32())
    d = S.prepare(c)[0]
    lat, frac = G.fcc(4.0)
    L, F, sp = G.supercell(lat, frac, [1] * 4, 2, 2, 2)
    comp = [(set(range(32)), {13: 16, 22: 16})]
    radii = G.distances_histogram(G.distance_matrix(L, F), 0.05, 0.25)
    o = G.prepare_interact(L, F, sp, comp, radii, {1: 1.0, 2: 0.5}, pair_weights=np.ones((2, 2, 2)))
    assert np.array_equal(d.species_packed, o.species_packed)
    assert np.array_equal(d.pairs, o.pairs)
    assert np.array_equal(d.prefactors, o.prefactors)
    assert np.array_equal(d.pair_weights, o.pair_weights)
    assert [tuple(w) for w in d.windows.tolist()] == o.bounds
    assert len(d.pairs) == 240 and np.bincount(d.pairs[:, 2]).tolist() == [192, 48]


# --------------------------------------------------------------------------- permutations
def test_permutations_match_oracle():
    k = json.load(open(os.path.join(GOLDEN, "permutation_kats.json")))
    for name, conf in k["configurations"].items():
        if name in k["num_permutations"]:
            assert N.num_permutations(conf) == k["num_permutations"][name]
    rng = np.random.default_rng(3)
    base = np.array([0] * 5 + [1] * 4 + [2] * 3 + [3] * 2, np.uint8)
    total = N.num_permutations(base)
    assert total == oracle.num_permutations(base)
    for r in rng.integers(1, total + 1, size=300):
        u = N.unrank_permutation(base, int(r))
        assert np.array_equal(u, oracle.unrank_permutation(base, int(r)))
        assert N.rank_permutation(u) == int(r)
    big = np.array([0] * 30 + [1] * 30 + [2] * 30, np.uint8)
    with pytest.raises(N.NativeError):
        N.num_permutations(big)


# --------------------------------------------------------------------------- parser
def code(res):
    assert isinstance(res, S.ParseError), res
    return res.key, res.code


def test_parse_defaults():
    """io/config/combined.h:38-39, shell_weights.h:75-83, arrays.h:103-107."""
    cfg = cases.fcc32()
    for k in ("shell_weights", "pair_weights", "iterations", "keep", "seed"):
        cfg.pop(k)
    c = S.parse_config(cfg)
    assert c.iterations == 500000 and c.chunk_size == 100000 and c.keep == 1
    assert list(c.shell_weights[0]) == list(range(1, len(c.shell_radii[0])))
    assert all(np.isclose(w, 1.0 / s) for s, w in c.shell_weights[0].items())
    K = 2
    assert np.array_equal(c.pair_weights[0][0], np.ones((K, K)) - np.eye(K))
    assert c.seed == [None]


def test_parse_errors_like_reference():
    assert code(S.parse_config({**cases.fcc32(), "bogus": 1})) == ("bogus", ParseErrorCode.bad_value)
    assert code(S.parse_config({**cases.fcc32(), "thread_config": 4})) == ("seed", ParseErrorCode.bad_value)
    assert code(S.parse_config({**cases.fcc32(), "keep": 0})) == ("keep", ParseErrorCode.bad_value)
    sys_seed = {**cases.settings_16(), "seed": 3}
    assert code(S.parse_config(sys_seed)) == ("seed", ParseErrorCode.bad_argument)
    split_one = {**cases.fcc32(), "sublattice_mode": "split"}
    assert code(S.parse_config(split_one)) == ("composition", ParseErrorCode.bad_value)
    bad_comp = {**cases.fcc32(), "composition": {"Ti": 16, "Al": 15}}
    assert code(S.parse_config(bad_comp)) == ("sites", ParseErrorCode.out_of_range)
    no_struct = {k: v for k, v in cases.fcc32().items() if k != "structure"}
    assert code(S.parse_config(no_struct)) == ("structure", ParseErrorCode.not_found)
    assert code(S.parse_config({**cases.fcc32(), "chunk_size": 10 ** 7})) == ("chunk_size", ParseErrorCode.out_of_range)
    assert code(S.parse_config({**cases.fcc32(), "shell_weights": {"0": 1.0}}))[0] == "shell_weights"
    sys_split = {**cases.rocksalt_split(), "iteration_mode": "systematic"}
    sys_split.pop("seed")
    assert code(S.parse_config(sys_split)) == ("iteration_mode", ParseErrorCode.bad_value)


def test_parse_systematic_iterations_and_seed_broadcast():
    c = S.parse_config(cases.settings_16())
    assert c.iterations == 12870
    c = S.parse_config(cases.rocksalt_split())
    assert c.seed == [3, 3]  # one seed copied to every sublattice (combined.h:62-65)


def test_parse_arrays_broadcast():
    cfg = {**cases.fcc32(), "target_objective": [[0.0, 0.1], [0.1, 0.0]], "prefactors": 0.5}
    c = S.parse_config(cfg)
    assert c.target_objective[0].shape == (2, 2, 2) and c.target_objective[0][1, 0, 1] == 0.1
    assert np.all(c.prefactors[0] == 0.5)
    bad = {**cases.fcc32(), "target_objective": np.zeros((3, 2, 2)).tolist()}
    assert code(S.parse_config(bad)) == ("target_objective", ParseErrorCode.bad_value)


def test_structure_sliced_like_reference():
    """core/structure.h sliced, as the reference's tests/test_structure.cpp:192-207 checks it: indices
    out of range and an empty selection are errors, repeated indices repeat the site."""
    from sqsgenerator_b200.core import Structure

    s = Structure(np.diag([1.0, 2.0, 3.0]), np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]]),
                  [11, 12, 13, 14])
    assert len(s.sliced(range(4))) == 4
    with pytest.raises(IndexError):
        s.sliced(range(-1, 4))
    with pytest.raises(IndexError):
        s.sliced(range(3, 6))
    with pytest.raises(ValueError):
        s.sliced([])
    r = s.sliced([1, 1, 1])
    assert r.species == [12, 12, 12]
    assert len({tuple(c) for c in r.frac_coords.tolist()}) == 1


def test_fcc_naive_shell_distances():
    """tests/test_structure.cpp:209-220 of the reference: the naive shell distances of an fcc 3x3x3 cell
    of one species (lattice constant 1) are 0, 1/sqrt(2), 1, sqrt(1.5), sqrt(2), sqrt(2.5), sqrt(3),
    sqrt(3.5), sqrt(4.5), sqrt(5.5) (its coordination numbers are checked in
    test_prefactors_and_pairs_match_oracle)."""
    L, F, Sp = N.supercell(np.eye(3), [[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]], [1, 1, 1, 1], 3, 3, 3)
    radii = N.distances_naive(N.distance_matrix(L, F), np.finfo(np.float64).eps, 1e-9)
    want = [0, 1 / np.sqrt(2), 1, np.sqrt(1.5), np.sqrt(2), np.sqrt(2.5), np.sqrt(3), np.sqrt(3.5), np.sqrt(4.5),
            np.sqrt(5.5)]
    assert np.allclose(np.asarray(radii), want, rtol=0, atol=1e-9)
