"""``parse_config``: the reference parameter schema turned into an ``SqsConfiguration``.

Restates ``include/sqsgen/io/config/combined.h:192-295`` and the per-key parsers it calls
(``composition.h``, ``shell_radii.h``, ``shell_weights.h``, ``arrays.h``, ``structure.h``), including
defaults and error keys/codes. Like the reference's Python binding, failures are *returned* as
``ParseError`` values. Geometry (supercell, distances, shells, prefactors) runs in the native library.
"""
from __future__ import annotations

import json
import numbers
import os
from typing import Any

import numpy as np

from . import _native
from .core import (SYMBOL_MAP, SYMBOLS, IterationMode, ParseError, ParseErrorCode, Prec, ShellRadiiDetection,
                   SqsConfiguration, Structure, Sublattice, SublatticeMode, dtype_of)

KNOWN_KEYS = (
    "iteration_mode", "sublattice_mode", "seed", "structure", "composition", "shell_radii", "shell_weights",
    "prefactors", "pair_weights", "target_objective", "iterations", "chunk_size", "thread_config", "keep",
    "max_results_per_objective", "atol", "rtol", "prec", "bin_width", "peak_isolation",
)
ITERATIONS_DEFAULT = 500000  # combined.h:38
CHUNK_SIZE_DEFAULT = 100000  # combined.h:39
ATOL_DEFAULT, RTOL_DEFAULT = 1.0e-3, 1.0e-5  # shell_radii.h:19-20
BIN_WIDTH_DEFAULT, PEAK_ISOLATION_DEFAULT = 0.05, 0.25  # shell_radii.h:21-22
U64_MAX = (1 << 64) - 1


class _Fail(Exception):
    def __init__(self, key, code, msg):
        super().__init__(msg)
        self.err = ParseError(key, msg, ParseErrorCode(code), None)


def _fail(key, code, msg):
    raise _Fail(key, code, msg)


def _enum(value, enum_cls, key, names):
    if isinstance(value, enum_cls):
        return value
    if isinstance(value, str):
        v = value.lower()
        if v in names:
            return enum_cls[names[v]]
        _fail(key, ParseErrorCode.bad_value, f"Invalid value for \"{key}\": {value!r}")
    try:
        return enum_cls(int(value))
    except (TypeError, ValueError):
        _fail(key, ParseErrorCode.type_error, f"Cannot interpret \"{key}\"")


def _structure(doc, T) -> tuple[Structure, tuple]:
    """io/config/structure.h:130-158."""
    if "structure" not in doc:
        _fail("structure", ParseErrorCode.not_found, "You need to specify a structure")
    s = doc["structure"]
    if not isinstance(s, dict):
        _fail("structure", ParseErrorCode.type_error, "\"structure\" must be a dictionary")
    if "file" in s:
        _fail("structure", ParseErrorCode.bad_argument, "structure files are not read by this build; pass "
              "lattice, coords and species")
    for k in ("lattice", "coords"):
        if k not in s:
            _fail(k, ParseErrorCode.not_found, f"Missing \"{k}\"")
    # a value that does not convert to the matrix type is a type error (the reference's get_as of an
    # Eigen matrix, structure.h:143-144)
    try:
        lattice = np.asarray(s["lattice"], dtype=T)
    except (TypeError, ValueError):
        lattice = None
    if lattice is None or lattice.shape != (3, 3):
        _fail("lattice", ParseErrorCode.type_error, "lattice must be a 3x3 matrix")
    try:
        coords = np.asarray(s["coords"], dtype=T)
    except (TypeError, ValueError):
        coords = None
    if coords is None or coords.ndim != 2 or coords.shape[1] != 3:
        _fail("coords", ParseErrorCode.type_error, "coords must be a N x 3 matrix")
    if "species" not in s:
        _fail("species", ParseErrorCode.not_found, "Missing \"species\"")
    sp = list(s["species"])
    if len(sp) != coords.shape[0]:
        _fail("species", ParseErrorCode.out_of_range,
              f"Number of coordinates ({coords.shape[0]}) does not match number of species {len(sp)}")
    species = []
    for x in sp:
        if isinstance(x, str):
            if x not in SYMBOL_MAP:
                _fail("species", ParseErrorCode.out_of_range, f"An atomic element with name \"{x}\" is not known to me")
            species.append(SYMBOL_MAP[x])
        else:
            z = int(x)
            if not 0 <= z < len(SYMBOLS):
                _fail("species", ParseErrorCode.out_of_range, f"An atomic element with ordinal number {z} is not known to me")
            species.append(z)
    supercell = tuple(int(v) for v in s.get("supercell", (1, 1, 1)))
    if len(supercell) != 3 or any(v < 0 for v in supercell):
        _fail("supercell", ParseErrorCode.out_of_range, "A supercell replication factor must be positive")
    return Structure(lattice, coords, species), supercell


def _sites(spec, species, remaining):
    """composition.h:33-95 — explicit indices, species symbol(s), or the remaining sites."""
    n = len(species)
    if spec is None:
        return sorted(remaining)
    if isinstance(spec, str):
        spec = [spec]
    spec = list(spec)
    if spec and all(isinstance(x, str) for x in spec):
        present = set(species)
        wanted = set()
        for s in spec:
            if s not in SYMBOL_MAP:
                _fail("sites", ParseErrorCode.out_of_range, f"An atomic element with name \"{s}\" is not known to me")
            z = SYMBOL_MAP[s]
            if z not in present:
                _fail("sites", ParseErrorCode.out_of_range,
                      f"The specified structure does not contain a site with species \"{s}\"")
            wanted.add(z)
        return [i for i in range(n) if species[i] in wanted]
    out = set()
    for i in spec:
        i = int(i)
        if not 0 <= i < n:
            _fail("sites", ParseErrorCode.out_of_range, f"Invalid index {i}, the specified structure contains {n} sites")
        out.add(i)
    if not out:
        _fail("sites", ParseErrorCode.out_of_range, "You cannot specify an empty slice")
    return sorted(out)


def _composition(doc, species, mode) -> list[Sublattice]:
    """composition.h:126-195."""
    if "composition" not in doc:
        _fail("composition", ParseErrorCode.not_found, "You need to specify a composition")
    comp = doc["composition"]
    if isinstance(comp, dict):
        if mode == SublatticeMode.split:
            _fail("composition", ParseErrorCode.bad_value,
                  "You have specified \"split\" mode but only specified one sublattice")
        comp = [comp]
    if not isinstance(comp, (list, tuple)) or not comp:
        _fail("composition", ParseErrorCode.out_of_range, "Could not parse a valid sublattice")
    out: list[Sublattice] = []
    occupied: set = set()
    for d in comp:
        if not isinstance(d, dict):
            _fail("composition", ParseErrorCode.bad_value, "the JSON value is not an object")
        remaining = set(range(len(species))) - occupied
        if not remaining:
            _fail("sites", ParseErrorCode.out_of_range, "There are no remaining species left for the sublattice")
        sites = _sites(d.get("sites"), species, remaining)
        for s in sites:
            if s in occupied:
                _fail("sites", ParseErrorCode.bad_value,
                      f"The site with index {s} is contained in more than one sublattice. Make sure that the "
                      "\"sites\" argument does not contain overlapping index ranges")
        dist: dict[int, int] = {}
        for k, v in d.items():
            if k not in SYMBOL_MAP:
                continue
            # the amount is read as an integer (composition.h:106): anything else is a type error
            if isinstance(v, (bool, np.bool_)) or not isinstance(v, (numbers.Real, np.number)):
                _fail("composition", ParseErrorCode.type_error,
                      f"The amount of \"{k}\" atoms must be an integer, not {v!r}")
            amount = int(v)
            if amount > len(sites) or amount < 0:
                _fail("composition", ParseErrorCode.bad_value,
                      f"You want to distribute {amount} \"{k}\" atoms on a sublattice with {len(sites)} sites")
            dist[SYMBOL_MAP[k]] = amount
        if not dist:
            _fail("composition", ParseErrorCode.out_of_range,
                  "You have not distributed any valid species on the (sub)lattice")
        if sum(dist.values()) != len(sites):
            _fail("sites", ParseErrorCode.out_of_range,
                  f"The total number of distributed atoms is {sum(dist.values())} but the sublattice contains "
                  f"{len(sites)} sites")
        out.append(Sublattice(sites, dict(sorted(dist.items()))))
        occupied |= set(sites)
    return out


def apply_composition(species, composition: list[Sublattice]) -> list[int]:
    """core/structure.h:390-396."""
    out = list(species)
    for sl in composition:
        it = iter(sl.sites)
        for z in sorted(sl.composition):
            for _ in range(sl.composition[z]):
                out[next(it)] = z
    return out


def _radii_for(doc, spec, structure: Structure, T):
    """shell_radii.h:27-71."""
    if isinstance(spec, str) or isinstance(spec, ShellRadiiDetection):
        mode = _enum(spec, ShellRadiiDetection, "shell_radii", {"naive": "naive", "peak": "peak"})
        D = structure.distance_matrix()
        if mode == ShellRadiiDetection.naive:
            return _native.distances_naive(D, float(doc.get("atol", ATOL_DEFAULT)), float(doc.get("rtol", RTOL_DEFAULT)))
        try:
            return _native.distances_histogram(D, float(doc.get("bin_width", BIN_WIDTH_DEFAULT)),
                                               float(doc.get("peak_isolation", PEAK_ISOLATION_DEFAULT)))
        except _native.NativeError as e:
            _fail("shell_radii", ParseErrorCode.bad_value, str(e))
    radii = [float(x) for x in spec]
    if not radii:
        _fail("shell_radii", ParseErrorCode.out_of_range, "You need to define at least one coordination shells")
    for r in radii:
        if r < 0:
            _fail("shell_radii", ParseErrorCode.bad_value, f"You cannot specify a shell radius that is less than 0 ({r})")
    arr = np.asarray(radii, dtype=T)
    if arr[0] != 0.0 and not abs(float(arr[0])) <= 1e-5:
        arr = np.concatenate([np.zeros(1, dtype=T), arr])
    return arr


def _weights_one(d, n_shells, T):
    """shell_weights.h:47-73."""
    if not isinstance(d, dict):
        _fail("shell_weights", ParseErrorCode.bad_value, "\"shell_weights\" must be an object")
    w = {}
    for k, v in d.items():
        try:
            s = int(k)
        except (TypeError, ValueError):
            _fail("shell_weights", ParseErrorCode.bad_value, f"Could not parse shell index: {k}")
        if s == 0:
            _fail("shell_weights", ParseErrorCode.bad_value, "There is no point in including self-interactions")
        if s >= n_shells:
            _fail("shell_weights", ParseErrorCode.out_of_range,
                  f"There are {n_shells} shells but you specified a shell index of {s}")
        w[s] = T(v)
    if not w:
        _fail("shell_weights", ParseErrorCode.out_of_range, "shell weights cannot be empty")
    return dict(sorted(w.items()))


def _array(key, value, S, K, T):
    """arrays.h:76-130 — scalar, K x K matrix (stacked per shell) or S x K x K cube."""
    a = np.asarray(value, dtype=T)
    if a.ndim == 0:
        return np.full((S, K, K), a, dtype=T)
    if a.ndim == 2:
        if a.shape != (K, K):
            _fail(key, ParseErrorCode.bad_value,
                  f"matrix has invalid size {a.shape[0]}x{a.shape[1]} but expected {K}x{K}")
        return np.stack([a] * S).astype(T)
    if a.ndim == 3:
        if a.shape != (S, K, K):
            _fail(key, ParseErrorCode.bad_value,
                  f"array has invalid size {'x'.join(map(str, a.shape))} but expected {S}x{K}x{K}")
        return a.copy()
    _fail(key, ParseErrorCode.bad_value, "Could not convert to 3D array")


def parse_config(config: dict[str, Any] | str) -> SqsConfiguration | ParseError:
    """Parse a reference-schema configuration (dict or JSON string)."""
    if isinstance(config, str):
        config = json.loads(config)
    try:
        return _parse(dict(config))
    except _Fail as f:
        return f.err


def _parse(doc: dict) -> SqsConfiguration:
    for k in doc:
        if not isinstance(k, str):
            _fail("", ParseErrorCode.type_error, "The configuration dictionary must only hold string keys")
        if k not in KNOWN_KEYS:
            _fail(k, ParseErrorCode.bad_value, f"Unknown parameter \"{k}\"")
    prec = _enum(doc.get("prec", Prec.double), Prec, "prec", {"double": "double", "single": "single"})
    T = dtype_of(prec)
    imode = _enum(doc.get("iteration_mode", IterationMode.random), IterationMode, "iteration_mode",
                  {"random": "random", "systematic": "systematic"})
    smode = _enum(doc.get("sublattice_mode", SublatticeMode.interact), SublatticeMode, "sublattice_mode",
                  {"interact": "interact", "split": "split"})
    base, supercell = _structure(doc, T)
    if imode == IterationMode.systematic and smode == SublatticeMode.split:
        _fail("iteration_mode", ParseErrorCode.bad_value,
              "It is not possible to do an exhaustive search on multiple sublattices in mode \"split\"")
    structure = base.supercell(*supercell)
    composition = _composition(doc, structure.species, smode)
    applied = structure.with_species(apply_composition(structure.species, composition))

    # shell radii: per (sub)lattice
    if smode == SublatticeMode.interact:
        spec = doc.get("shell_radii", "peak")
        radii = [_radii_for(doc, spec, structure, T)]
        structs = [applied]
    else:
        structs = [applied.sliced(sl.sites) for sl in composition]
        if "shell_radii" in doc:
            spec = doc["shell_radii"]
            if not isinstance(spec, (list, tuple)):
                _fail("shell_radii", ParseErrorCode.type_error,
                      "You want to run a split sublattice mode, and did not specify valid modes. You have to "
                      "specify the shell radii per sublattice")
            if len(spec) != len(composition):
                _fail("shell_radii", ParseErrorCode.bad_value, "one shell radii entry per sublattice is required")
            radii = [_radii_for(doc, s, structure.sliced(sl.sites), T) for s, sl in zip(spec, composition)]
        else:
            radii = [_radii_for(doc, "peak", structure.sliced(sl.sites), T) for sl in composition]

    # iterations (combined.h:79-100)
    if imode == IterationMode.systematic:
        if len(composition) != 1:
            _fail("iterations", ParseErrorCode.bad_value, "In \"systematic\" iteration mode only one sublattice is allowed")
        sub = [applied.species[i] for i in composition[0].sites]
        zs = sorted(set(sub))
        packed = np.array([zs.index(z) for z in sub], dtype=np.uint8)
        try:
            iterations = _native.num_permutations(packed)
        except _native.NativeError:
            _fail("iterations", ParseErrorCode.bad_value,
                  "The number of permutations to test is too large. I'm a pretty fast program, but this is too "
                  "much even for me ;=)")
    else:
        iterations = int(doc.get("iterations", ITERATIONS_DEFAULT))
        if iterations < 0 or iterations > U64_MAX:
            _fail("iterations", ParseErrorCode.bad_value, "iterations must fit an unsigned 64-bit integer")

    # seed (combined.h:47-77)
    n_sl = 1 if smode == SublatticeMode.interact else len(composition)
    if "seed" in doc:
        if imode == IterationMode.systematic:
            _fail("seed", ParseErrorCode.bad_argument,
                  "You cannot specify a seed if you have set the iteration mode to \"systematic\". The seed is only "
                  "used for random iterations, but in systematic mode there is no randomness involved.")
        s = doc["seed"]
        if isinstance(s, (list, tuple)):
            if len(s) != n_sl:
                _fail("seed", ParseErrorCode.bad_value,
                      f"The number of seeds provided ({len(s)}) does not match the number of sublattices ({n_sl})")
            seed = [None if x is None else int(x) for x in s]
        else:
            seed = [int(s)] * n_sl
    else:
        seed = [None] * n_sl

    # shell weights (shell_weights.h:86-118)
    if "shell_weights" not in doc:
        weights = [{i: T(T(1.0) / T(i)) for i in range(1, len(r))} for r in radii]
    else:
        sw = doc["shell_weights"]
        if smode == SublatticeMode.interact:
            weights = [_weights_one(sw, len(radii[0]), T)]
        elif isinstance(sw, dict):
            weights = [_weights_one(sw, len(r), T) for r in radii]
        elif isinstance(sw, (list, tuple)):
            if len(sw) != len(radii):
                _fail("shell_weights", ParseErrorCode.bad_value, "one shell weights entry per sublattice is required")
            weights = [_weights_one(w, len(r), T) for w, r in zip(sw, radii)]
        else:
            _fail("shell_weights", ParseErrorCode.bad_value, "Cannot interpret value")

    # prefactors / pair weights / targets (arrays.h:132-190)
    def per_sublattice(key):
        if key not in doc:
            return [None] * len(structs)
        v = doc[key]
        if smode == SublatticeMode.split:
            if not isinstance(v, (list, tuple)):
                _fail(key, ParseErrorCode.type_error,
                      "You have specified \"split\" mode. In split mode array type parameter must be specified "
                      "per sublattice")
            if len(v) != len(structs):
                _fail(key, ParseErrorCode.bad_value, "one entry per sublattice is required")
            return list(v)
        return [v]

    prefactors, pair_weights, targets = [], [], []
    for st, r, w, pf, pw, tg in zip(structs, radii, weights, per_sublattice("prefactors"),
                                    per_sublattice("pair_weights"), per_sublattice("target_objective")):
        S, K = len(w), st.num_species
        if pf is None:
            sm = st.shell_matrix(r)
            prefactors.append(_native.prefactors(sm, list(w.keys()), st.species, dtype=T))
        else:
            prefactors.append(_array("prefactors", pf, S, K, T))
        if pw is None:
            pair_weights.append(np.stack([np.ones((K, K), dtype=T) - np.eye(K, dtype=T)] * S).astype(T))
        else:
            pair_weights.append(_array("pair_weights", pw, S, K, T))
        targets.append(np.zeros((S, K, K), dtype=T) if tg is None else _array("target_objective", tg, S, K, T))

    # chunk size (combined.h:122-136)
    chunk = int(doc.get("chunk_size", min(iterations, CHUNK_SIZE_DEFAULT)))
    if chunk > iterations:
        _fail("chunk_size", ParseErrorCode.out_of_range,
              f"\"chunk_size\" was set to {chunk} and iterations set to {iterations}")
    # thread config (combined.h:102-120)
    tc = doc.get("thread_config", os.cpu_count() or 1)
    thread_config = [int(x) for x in tc] if isinstance(tc, (list, tuple)) else [int(tc)]
    if any(t == 0 for t in thread_config) and not isinstance(tc, (list, tuple)):
        _fail("thread_config", ParseErrorCode.bad_value, "The number of threads cannot be set to 0")
    keep = int(doc.get("keep", 1))
    if keep == 0:
        _fail("keep", ParseErrorCode.bad_value, "The number of best kept structures must be greater than 0")
    mrpo = doc.get("max_results_per_objective")
    if mrpo is not None:
        mrpo = int(mrpo)
        if mrpo <= 0:
            _fail("max_results_per_objective", ParseErrorCode.bad_value,
                  "The number of structures per objective must be a positive integer number")
    if any(s is not None for s in seed) and any(t > 1 for t in thread_config):
        _fail("seed", ParseErrorCode.bad_value,
              "A random seed is set but the thread configuration specifies more than 1 thread; seeded runs "
              "require (currently) exactly 1 thread for reproducibility")
    return SqsConfiguration(prec, smode, imode, seed, base, supercell, composition, radii, weights, prefactors,
                            pair_weights, targets, iterations, chunk, thread_config, keep, mrpo)
