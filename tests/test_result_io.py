"""Result packs, configurations and structures written and read in the reference's msgpack layout.

The CPU tests build packs from synthetic results (species drawn from the configuration's composition,
random SRO cubes) and check the round trip and the document layout of include/sqsgen/io/json.h:120-287.
The GPU test follows python/tests/test_core.py:132-175 of the reference (``test_structure_pack_io``):
optimise, write ``pack.bytes()``, load from bytes and from a file, compare configuration by configuration.
"""
from __future__ import annotations

import math
import os
import tempfile

import msgpack
import numpy as np
import pytest

import sqsgenerator_b200 as S
from sqsgenerator_b200.core import SqsResult, SqsResultPack, SqsResultSplit, SqsStatistics

import cases


def _synthetic_pack(settings, n=40, seed=5):
    c = S.parse_config(settings)
    assert not isinstance(c, S.ParseError), c
    data = S.prepare(c)
    T = np.float64 if int(c.prec) == 1 else np.float32
    rng = np.random.default_rng(seed)
    levels = np.sort(rng.random(4)).astype(T)
    results = []
    for r in range(n):
        per = []
        for d in data:
            z = np.asarray(d.structure.species)
            S_, K = d.prefactors.shape[0], d.prefactors.shape[1]
            per.append(SqsResult(T(rng.choice(levels)), rng.permutation(z).tolist(),
                                 rng.standard_normal((S_, K, K)).astype(T), d))
        obj = T(levels[r % len(levels)])
        if c.sublattice_mode == S.SublatticeMode.interact:
            per[0].objective = obj
            results.append(per[0])
        else:
            full = c.structure()
            from sqsgenerator_b200.config import apply_composition
            full = full.with_species(apply_composition(full.species, c.composition))
            results.append(SqsResultSplit(obj, per, full, [sl.sites for sl in c.composition]))
    stats = SqsStatistics(123, 4, 77, float(levels[0]), {"total": 9, "chunk_setup": 1, "loop": 7, "comm": 1})
    return SqsResultPack(c, results, stats)


def _by_species(pack):
    return {"".join(map(str, r.species)): r for _, group in pack for r in group}


def _same_pack(a, b):
    assert a.num_results() == b.num_results()
    assert a.num_objectives() == b.num_objectives()
    assert [o for o, _ in a] == [o for o, _ in b]
    for (_, ga), (_, gb) in zip(a, b):
        for ra, rb in zip(ga, gb):
            assert ra.objective == rb.objective
            assert list(ra.species) == list(rb.species)
            if isinstance(ra, SqsResultSplit):
                for sa, sb in zip(ra.sublattices, rb.sublattices):
                    assert sa.objective == sb.objective and list(sa.species) == list(sb.species)
                    np.testing.assert_array_equal(sa.sro(), sb.sro())
            else:
                np.testing.assert_array_equal(ra.sro(), rb.sro())
            np.testing.assert_array_equal(ra.structure().frac_coords, rb.structure().frac_coords)
    sa, sb = a.statistics, b.statistics
    assert (sa.finished, sa.working, sa.best_rank, sa.best_objective, sa.timings) == \
        (sb.finished, sb.working, sb.best_rank, sb.best_objective, sb.timings)


@pytest.mark.parametrize("prec", ["single", "double"])
@pytest.mark.parametrize("make", [cases.fcc32, cases.rocksalt_split, cases.quinary])
def test_pack_round_trip(make, prec):
    pack = _synthetic_pack(make(prec))
    loaded = S.load_result_pack(pack.bytes(), S.Prec[prec])
    _same_pack(pack, loaded)
    assert loaded.config.sublattice_mode == pack.config.sublattice_mode
    assert loaded.config.iteration_mode == pack.config.iteration_mode
    assert loaded.config.keep == pack.config.keep
    assert loaded.config.shell_weights == [{k: float(v) for k, v in w.items()} for w in pack.config.shell_weights]
    for x, y in zip(loaded.config.pair_weights, pack.config.pair_weights):
        np.testing.assert_array_equal(x, y)


def test_pack_round_trip_through_a_file():
    pack = _synthetic_pack(cases.fcc32("double"))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "pack.msgpack")
        S.dump_result_pack(pack, path)
        loaded = S.load_result_pack(path, S.Prec.double)
    _same_pack(pack, loaded)


def test_document_layout_follows_the_reference():
    pack = _synthetic_pack(cases.quinary("double", cells=(2, 2, 2)), n=7)
    doc = msgpack.unpackb(pack.bytes(), raw=False, strict_map_key=False)
    assert set(doc) == {"statistics", "config", "results"}
    st = doc["statistics"]
    assert set(st) == {"best_objective", "best_rank", "finished", "working", "timings"}
    # std::map<Timing, ns> with an enum key: [name, value] pairs in enum order
    assert st["timings"] == [["total", 9], ["chunk_setup", 1], ["loop", 7], ["comm", 1]]
    cfg = doc["config"]
    assert cfg["sublattice_mode"] == "interact" and cfg["iteration_mode"] == "random"
    assert set(cfg["structure"]) == {"lattice", "species", "coords", "supercell"}
    assert cfg["structure"]["supercell"] == [2, 2, 2]
    comp = cfg["composition"][0]
    assert comp["sites"] == sorted(comp["sites"])
    assert all(isinstance(p, list) and len(p) == 2 for p in comp["composition"])
    assert [p[0] for p in comp["composition"]] == sorted(p[0] for p in comp["composition"])
    assert cfg["shell_weights"] == [[[1, 1.0], [2, 0.5], [3, 0.25]]]
    assert np.asarray(cfg["pair_weights"][0]).shape == (3, 5, 5)
    assert cfg["max_results_per_objective"] is None
    assert [r["objective"] for r in doc["results"]] == sorted(r["objective"] for r in doc["results"])
    r0 = doc["results"][0]
    assert set(r0) == {"objective", "species", "sro"}
    # SRO: Eigen::Tensor column-major data, first index fastest
    best = pack.best()
    assert r0["sro"]["shape"] == list(best.sro().shape)
    assert r0["sro"]["data"] == best.sro().ravel(order="F").tolist()


def test_split_document_has_sublattices():
    pack = _synthetic_pack(cases.rocksalt_split("single"), n=3)
    doc = msgpack.unpackb(pack.bytes(), raw=False, strict_map_key=False)
    assert doc["config"]["sublattice_mode"] == "split"
    for r in doc["results"]:
        assert set(r) == {"objective", "sublattices"}
        assert len(r["sublattices"]) == 2
        assert all(set(x) == {"objective", "species", "sro"} for x in r["sublattices"])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["single", "double"])
def test_structure_pack_io(prec):
    results = S.optimize(S.parse_config(cases.settings_16(prec)))
    assert type(S.load_result_pack(results.bytes(), S.Prec[prec])) is type(results)
    with tempfile.NamedTemporaryFile(mode="wb") as f:
        f.write(results.bytes())
        f.flush()
        loaded = S.load_result_pack(f.name, S.Prec[prec])
    rl, rr = _by_species(loaded), _by_species(results)
    assert len(rr) == len(rl) == loaded.num_results() == results.num_results() == 12870
    assert set(rl) == set(rr)
    for key, a in rr.items():
        b = rl[key]
        assert math.isclose(a.objective, b.objective)
        assert np.allclose(a.sro(), b.sro())
        sa, sb = a.structure(), b.structure()
        np.testing.assert_allclose(sa.lattice, sb.lattice)
        np.testing.assert_allclose(sa.frac_coords, sb.frac_coords)
        assert list(sa.species) == list(sb.species)


@pytest.mark.parametrize("make", [cases.fcc32, cases.rocksalt_split])
def test_configuration_bytes_and_json(make):
    import json

    c = S.parse_config(make("double"))
    back = S.SqsConfiguration.from_bytes(c.bytes(), S.Prec.double)
    assert back.sublattice_mode == c.sublattice_mode and back.iteration_mode == c.iteration_mode
    assert back.supercell == tuple(c.supercell) and back.keep == c.keep and back.seed == list(c.seed)
    assert [sl.sites for sl in back.composition] == [sorted(sl.sites) for sl in c.composition]
    assert [sl.composition for sl in back.composition] == [sl.composition for sl in c.composition]
    for x, y in zip(back.target_objective, c.target_objective):
        np.testing.assert_array_equal(x, y)
    doc = json.loads(c.json())
    assert list(doc) == sorted(doc)  # nlohmann::json keeps object keys sorted
    assert set(doc) == {"sublattice_mode", "iteration_mode", "seed", "structure", "composition", "shell_radii",
                        "shell_weights", "prefactors", "pair_weights", "target_objective", "iterations",
                        "chunk_size", "thread_config", "keep", "max_results_per_objective"}
    assert " " not in c.json()  # compact dump
    # the configuration's prepared data is the same after the round trip
    for a, b in zip(S.prepare(c), S.prepare(back)):
        np.testing.assert_array_equal(a.pairs, b.pairs)
        np.testing.assert_array_equal(a.species_packed, b.species_packed)


def test_structure_bytes_round_trip():
    s = S.parse_config(cases.rocksalt_split("single")).structure()
    doc = msgpack.unpackb(s.bytes(), raw=False)
    assert list(doc) == ["frac_coords", "lattice", "pbc", "species"]
    back = S.Structure.from_bytes(s.bytes(), S.Prec.single)
    assert back.lattice.dtype == np.float32
    np.testing.assert_array_equal(back.lattice, s.lattice)
    np.testing.assert_array_equal(back.frac_coords, s.frac_coords)
    assert back.species == s.species and back.pbc == tuple(s.pbc)


def _nlohmann_include():
    import glob
    import sys as _sys

    for root in {_sys.prefix, os.path.dirname(os.path.dirname(np.__file__))}:
        for hit in glob.glob(os.path.join(root, "**", "nlohmann", "json.hpp"), recursive=True):
            return os.path.dirname(os.path.dirname(hit))
    return None


@pytest.mark.parametrize("settings", ["interact_double", "interact_single", "split_double", "split_single"])
def test_pack_reads_with_nlohmann_from_msgpack(settings, tmp_path):
    """The bytes of pack.bytes() decode with nlohmann::json::from_msgpack (the call the reference's loader
    uses, python/extension/sqsgen.cpp:38-56) and read with the reference's keys and value types
    (tests/pack_reader.cpp follows include/sqsgen/io/json.h:120-287)."""
    inc = _nlohmann_include()
    if inc is None:
        pytest.skip("nlohmann/json.hpp is not installed on this machine")
    exe = tmp_path / "pack_reader"
    src = os.path.join(os.path.dirname(__file__), "pack_reader.cpp")
    import subprocess

    subprocess.run(["g++", "-std=c++20", "-O1", "-I", inc, src, "-o", str(exe)], check=True)
    mode, prec = settings.split("_")
    cfg = cases.settings_16(prec) if mode == "interact" else cases.rocksalt_split(prec, iterations=1000)
    pack = _synthetic_pack(cfg, n=25)
    path = tmp_path / "pack.msgpack"
    path.write_bytes(pack.bytes())
    out = subprocess.run([str(exe), str(path), prec], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    n_results, n_sro = (int(x) for x in out.stdout.split()[1::2])
    assert n_results == pack.num_results()
    per = sum(d.prefactors.size for d in S.prepare(pack.config))
    assert n_sro == n_results * per
