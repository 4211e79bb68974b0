"""Result packs on disk in the reference's format.

The reference stores a result pack as the msgpack encoding of one JSON document
``{"statistics", "config", "results"}`` (``include/sqsgen/io/json.h:120-287``; written and read with
``nlohmann::json::to_msgpack`` / ``from_msgpack`` in ``python/extension/sqsgen.cpp:29-80``):

- ``std::map`` values whose keys are not strings (composition ``Z -> count``, shell weights
  ``shell -> weight``, timings ``Timing -> ns``) are arrays of ``[key, value]`` pairs in key order;
  enums are their names (``"interact"``, ``"random"``, ``"total"``, ...);
- ``results`` is the flattened list, ascending by objective; an interact result is
  ``{"objective", "species", "sro": {"shape": [S, K, K], "data": [...]}}`` with the SRO cube in the
  column-major order of an ``Eigen::Tensor`` (first index fastest); a split result is
  ``{"objective", "sublattices": [interact results]}``;
- cubes of the configuration (prefactors, pair weights, targets) are nested ``[S][K][K]`` lists.

``dump_result_pack`` writes that document; ``load_result_pack`` reads it back into a
``SqsResultPack`` (the precision is not stored, as in the reference, and is passed in). Structures and
configurations have the same ``bytes()`` / ``from_bytes`` pair, and configurations a compact
``json()``, with the documents of ``io/json.h:138-212``. Object keys are written sorted, as
``nlohmann::json`` keeps them.
"""
from __future__ import annotations

import json
import os
from typing import Any

import msgpack
import numpy as np

from .config import apply_composition
from .core import (IterationMode, Prec, SqsConfiguration, SqsResult, SqsResultPack, SqsResultSplit, SqsStatistics,
                   Structure, Sublattice, SublatticeMode, dtype_of)
from .optimize import TIMING_NAMES, prepare


def _pairs(mapping) -> list:
    return [[int(k), v] for k, v in sorted(mapping.items())]


def _from_pairs(pairs, key=int, value=lambda v: v) -> dict:
    return {key(k): value(v) for k, v in pairs}


def _cube(a) -> list:
    return np.asarray(a).tolist()


def _sro_doc(cube: np.ndarray) -> dict:
    cube = np.asarray(cube)
    return {"shape": [int(x) for x in cube.shape], "data": [float(x) for x in cube.ravel(order="F")]}


def _sro_cube(doc: dict, dtype) -> np.ndarray:
    shape = tuple(int(x) for x in doc["shape"])
    return np.asarray(doc["data"], dtype=dtype).reshape(shape, order="F")


def config_to_doc(c: SqsConfiguration) -> dict:
    """``adl_serializer<configuration<T>>::to_json`` (include/sqsgen/io/json.h:176-195)."""
    s = c.structure_config
    return {
        "sublattice_mode": c.sublattice_mode.name,
        "iteration_mode": c.iteration_mode.name,
        "seed": [None if x is None else int(x) for x in c.seed],
        "structure": {"lattice": np.asarray(s.lattice).tolist(), "species": [int(z) for z in s.species],
                      "coords": np.asarray(s.frac_coords).tolist(), "supercell": [int(x) for x in c.supercell]},
        "composition": [{"sites": sorted(int(i) for i in sl.sites), "composition": _pairs(sl.composition)}
                        for sl in c.composition],
        "shell_radii": [[float(r) for r in radii] for radii in c.shell_radii],
        "shell_weights": [[[int(k), float(v)] for k, v in sorted(w.items())] for w in c.shell_weights],
        "prefactors": [_cube(x) for x in c.prefactors],
        "pair_weights": [_cube(x) for x in c.pair_weights],
        "target_objective": [_cube(x) for x in c.target_objective],
        "iterations": None if c.iterations is None else int(c.iterations),
        "chunk_size": int(c.chunk_size),
        "thread_config": [int(x) for x in c.thread_config],
        "keep": int(c.keep),
        "max_results_per_objective": None if c.max_results_per_objective is None
        else int(c.max_results_per_objective),
    }


def config_from_doc(doc: dict, prec: Prec) -> SqsConfiguration:
    T = dtype_of(prec)
    st = doc["structure"]
    structure = Structure(np.asarray(st["lattice"], dtype=T), np.asarray(st["coords"], dtype=T),
                          [int(z) for z in st["species"]])
    return SqsConfiguration(
        prec=Prec(prec),
        sublattice_mode=SublatticeMode[doc["sublattice_mode"]],
        iteration_mode=IterationMode[doc["iteration_mode"]],
        seed=list(doc["seed"]),
        structure_config=structure,
        supercell=tuple(int(x) for x in st["supercell"]),
        composition=[Sublattice([int(i) for i in sl["sites"]], _from_pairs(sl["composition"], int, int))
                     for sl in doc["composition"]],
        shell_radii=[np.asarray(r, dtype=T) for r in doc["shell_radii"]],
        shell_weights=[_from_pairs(w, int, float) for w in doc["shell_weights"]],
        prefactors=[np.asarray(x, dtype=T) for x in doc["prefactors"]],
        pair_weights=[np.asarray(x, dtype=T) for x in doc["pair_weights"]],
        target_objective=[np.asarray(x, dtype=T) for x in doc["target_objective"]],
        iterations=doc["iterations"],
        chunk_size=int(doc["chunk_size"]),
        thread_config=[int(x) for x in doc["thread_config"]],
        keep=int(doc["keep"]),
        max_results_per_objective=doc["max_results_per_objective"],
    )


def pack_to_doc(pack: SqsResultPack) -> dict:
    """``adl_serializer<sqs_result_pack<T, Mode>>::to_json`` (include/sqsgen/io/json.h:264-275)."""
    st = pack.statistics
    results: list[Any] = []
    for _, group in pack:
        for r in group:
            if isinstance(r, SqsResultSplit):
                results.append({"objective": float(r.objective),
                                "sublattices": [{"objective": float(x.objective), "species": [int(z) for z in x.species],
                                                 "sro": _sro_doc(x.sro())} for x in r.sublattices]})
            else:
                results.append({"objective": float(r.objective), "species": [int(z) for z in r.species],
                                "sro": _sro_doc(r.sro())})
    return {
        "statistics": {"best_objective": float(st.best_objective), "best_rank": int(st.best_rank),
                       "finished": int(st.finished), "working": int(st.working),
                       "timings": [[name, int(st.timings.get(name, 0))] for name in TIMING_NAMES]},
        "config": config_to_doc(pack.config),
        "results": results,
    }


def _sorted(doc):
    """Object keys in sorted order at every level, as nlohmann::json (a std::map) writes them."""
    if isinstance(doc, dict):
        return {k: _sorted(doc[k]) for k in sorted(doc)}
    if isinstance(doc, list):
        return [_sorted(x) for x in doc]
    return doc


def _pack(doc) -> bytes:
    return msgpack.packb(_sorted(doc), use_bin_type=True)


def _unpack(data) -> dict:
    return msgpack.unpackb(bytes(data), raw=False, strict_map_key=False)


def structure_to_doc(s: Structure) -> dict:
    """``adl_serializer<core::structure<T>>`` (include/sqsgen/io/json.h:138-156)."""
    return {"lattice": np.asarray(s.lattice).tolist(), "species": [int(z) for z in s.species],
            "frac_coords": np.asarray(s.frac_coords).tolist(), "pbc": [bool(x) for x in s.pbc]}


def structure_from_doc(doc: dict, prec: Prec) -> Structure:
    T = dtype_of(prec)
    return Structure(np.asarray(doc["lattice"], dtype=T), np.asarray(doc["frac_coords"], dtype=T).reshape(-1, 3),
                     [int(z) for z in doc["species"]], tuple(bool(x) for x in doc["pbc"]))


def dump_structure(s: Structure) -> bytes:
    """``Structure.bytes()`` of the reference (python/extension/sqsgen.cpp:182)."""
    return _pack(structure_to_doc(s))


def load_structure(data: bytes, prec: Prec = Prec.double) -> Structure:
    return structure_from_doc(_unpack(data), prec)


def dump_configuration(c: SqsConfiguration) -> bytes:
    """``SqsConfiguration.bytes()`` of the reference (python/extension/sqsgen.cpp:222)."""
    return _pack(config_to_doc(c))


def configuration_json(c: SqsConfiguration) -> str:
    """``SqsConfiguration.json()`` of the reference: the compact dump, keys sorted
    (python/extension/sqsgen.cpp:223-227)."""
    return json.dumps(_sorted(config_to_doc(c)), separators=(",", ":"))


def load_configuration(data: bytes, prec: Prec = Prec.single) -> SqsConfiguration:
    return config_from_doc(_unpack(data), prec)


def dump_result_pack(pack: SqsResultPack, path: str | os.PathLike | None = None) -> bytes:
    """The msgpack bytes of the pack's document; also written to ``path`` when given."""
    data = _pack(pack_to_doc(pack))
    if path is not None:
        with open(path, "wb") as f:
            f.write(data)
    return data


def load_result_pack(data: bytes | str | os.PathLike, prec: Prec = Prec.single) -> SqsResultPack:
    """Read a pack written by ``dump_result_pack`` (or the reference) from bytes or a file path; like the
    reference's ``load_result_pack(data, prec)`` the precision is given by the caller."""
    if not isinstance(data, (bytes, bytearray)):
        with open(data, "rb") as f:
            data = f.read()
    doc = _unpack(data)
    config = config_from_doc(doc["config"], prec)
    parts = prepare(config)
    T = dtype_of(config.prec)
    full = config.structure()
    full = full.with_species(apply_composition(full.species, config.composition))
    results = []
    for r in doc["results"]:
        if "sublattices" in r:
            subs = [SqsResult(T(x["objective"]), list(x["species"]), _sro_cube(x["sro"], T), d)
                    for x, d in zip(r["sublattices"], parts)]
            results.append(SqsResultSplit(T(r["objective"]), subs, full, [sl.sites for sl in config.composition]))
        else:
            results.append(SqsResult(T(r["objective"]), list(r["species"]), _sro_cube(r["sro"], T), parts[0]))
    s = doc["statistics"]
    stats = SqsStatistics(int(s["finished"]), int(s["working"]), int(s["best_rank"]), float(s["best_objective"]),
                          _from_pairs(s["timings"], str, int))
    return SqsResultPack(config, results, stats)
