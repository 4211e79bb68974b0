"""Value types of the Python mirror of the reference API.

Mirrors the objects ``sqsgenerator.core`` exposes (``python/sqsgenerator/core/_core.pyi`` in the
reference): enums, ``ParseError``, ``Structure``, ``SqsConfiguration``, ``SqsResult`` and
``SqsResultPack``. Result accessors follow ``include/sqsgen/core/results.h:142-283``.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import Iterator

import numpy as np

from . import _native

# Element symbols by atomic number (index = Z); "0" is the vacancy (include/sqsgen/core/atom.h:20).
SYMBOLS = (
    "0 H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
    "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb "
    "Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr Rf "
    "Db Sg Bh Hs Mt Ds Rg Cn Nh Fl"
).split()
SYMBOL_MAP = {s: z for z, s in enumerate(SYMBOLS)}


class Prec(enum.IntEnum):
    single = 0
    double = 1


class IterationMode(enum.IntEnum):
    random = 0
    systematic = 1


class SublatticeMode(enum.IntEnum):
    interact = 0
    split = 1


class ShellRadiiDetection(enum.IntEnum):
    naive = 0
    peak = 1


class LogLevel(enum.IntEnum):
    trace = 0
    debug = 1
    info = 2
    warn = 3
    error = 4


class ParseErrorCode(enum.IntEnum):
    """``include/sqsgen/io/parsing.h:19-26``."""

    unknown = -1
    not_found = 0
    type_error = 1
    out_of_range = 2
    bad_value = 3
    bad_argument = 4


@dataclass
class ParseError:
    """Returned (not raised) by ``parse_config`` like the reference's ``_core.parse_config``."""

    key: str
    msg: str
    code: ParseErrorCode
    parameter: str | None = None

    def __str__(self) -> str:
        return f"ParseError(key={self.key!r}, code={self.code.name}, msg={self.msg!r})"


def dtype_of(prec: Prec):
    return np.float64 if prec == Prec.double else np.float32


@dataclass
class Structure:
    """A periodic structure: lattice rows, fractional coordinates, atomic numbers."""

    lattice: np.ndarray
    frac_coords: np.ndarray
    species: list[int]
    pbc: tuple = (True, True, True)

    def __len__(self) -> int:
        return len(self.species)

    def __iter__(self) -> Iterator[tuple[int, np.ndarray, int]]:
        for i, (c, z) in enumerate(zip(self.frac_coords, self.species)):
            yield i, c, z

    @property
    def num_species(self) -> int:
        return len(set(self.species))

    @property
    def symbols(self) -> list[str]:
        return [SYMBOLS[z] for z in self.species]

    def supercell(self, a: int, b: int, c: int) -> "Structure":
        lo, fo, so = _native.supercell(self.lattice, self.frac_coords, self.species, a, b, c,
                                       dtype=self.lattice.dtype)
        return Structure(lo, fo, so.tolist(), self.pbc)

    def distance_matrix(self) -> np.ndarray:
        return _native.distance_matrix(self.lattice, self.frac_coords, dtype=self.lattice.dtype)

    def shell_matrix(self, shell_radii, atol=None, rtol=1.0e-9) -> np.ndarray:
        atol = np.finfo(self.lattice.dtype).eps if atol is None else atol
        return _native.shell_matrix(self.distance_matrix(), np.asarray(shell_radii, self.lattice.dtype),
                                    atol, rtol)

    def sliced(self, sites) -> "Structure":
        sites = list(sites)
        if not sites:
            raise ValueError("Cannot create a structure without atoms")
        for i in sites:
            if i < 0 or i >= len(self):
                raise IndexError(f"index out of range 0 <= {i} < {len(self)}")
        return Structure(self.lattice.copy(), self.frac_coords[sites].copy(), [self.species[i] for i in sites],
                         self.pbc)

    def with_species(self, species) -> "Structure":
        if len(species) != len(self):
            raise ValueError("Species size mismatch")
        return Structure(self.lattice.copy(), self.frac_coords.copy(), list(species), self.pbc)

    def bytes(self) -> bytes:
        from .io import dump_structure

        return dump_structure(self)

    @staticmethod
    def from_bytes(data: bytes, prec: Prec = Prec.double) -> "Structure":
        from .io import load_structure

        return load_structure(data, prec)


@dataclass
class Sublattice:
    sites: list[int]
    composition: dict[int, int]


@dataclass
class SqsConfiguration:
    """The parsed configuration (``include/sqsgen/core/config.h:32-48``)."""

    prec: Prec
    sublattice_mode: SublatticeMode
    iteration_mode: IterationMode
    seed: list
    structure_config: Structure
    supercell: tuple
    composition: list[Sublattice]
    shell_radii: list[np.ndarray]
    shell_weights: list[dict]
    prefactors: list[np.ndarray]
    pair_weights: list[np.ndarray]
    target_objective: list[np.ndarray]
    iterations: int
    chunk_size: int
    thread_config: list[int]
    keep: int
    max_results_per_objective: int | None

    def structure(self) -> Structure:
        a, b, c = self.supercell
        return self.structure_config.supercell(a, b, c)

    def bytes(self) -> bytes:
        from .io import dump_configuration

        return dump_configuration(self)

    def json(self) -> str:
        from .io import configuration_json

        return configuration_json(self)

    @staticmethod
    def from_bytes(data: bytes, prec: Prec = Prec.single) -> "SqsConfiguration":
        from .io import load_configuration

        return load_configuration(data, prec)


@dataclass
class SqsStatistics:
    """``sqs_statistics_data`` (include/sqsgen/types.h:197-206)."""

    finished: int = 0
    working: int = 0
    best_rank: int = 0
    best_objective: float = float("inf")
    timings: dict = field(default_factory=dict)


@dataclass
class OptimizationData:
    """Per-(sub)lattice data of ``optimization_config_data`` (core/optimization_config.h:33-48)."""

    structure: Structure            # composition applied, original site order
    sorted_structure: Structure     # sites sorted by sublattice
    sort_order: np.ndarray          # sorted position -> original site
    windows: np.ndarray             # shuffle windows (sorted order)
    species_packed: np.ndarray      # dense species indices, sorted order
    species_map: dict               # Z -> dense index
    species_rmap: dict              # dense index -> Z
    shell_map: dict                 # shell id -> dense index
    pairs: np.ndarray               # (P, 3) i < j, dense shell
    prefactors: np.ndarray
    pair_weights: np.ndarray        # scaled by the shell weights
    target: np.ndarray
    shell_radii: np.ndarray
    shell_weights: dict
    sublattices: list
    lattice: np.ndarray | None = None  # (N, 4) per sorted site: unit-cell site, cell indices a, b, c
    cells: tuple = (0, 0, 0)            # supercell repetitions along the three lattice vectors


class SqsResult:
    """One configuration (``sqs_result_wrapper<T, INTERACT>``, core/results.h:142-228)."""

    def __init__(self, objective, species, sro, data: OptimizationData, rank_id=None):
        self.objective = objective
        self.species = species          # atomic numbers, original site order of the structure
        self._sro = sro                 # (S, K, K)
        self._data = data
        self.id = rank_id

    def sro(self, *args):
        """Without arguments the (S, K, K) cube; sro(shell, i, j) / sro(shell) / sro(i, j) like the
        reference's overloads (results.h:164-214)."""
        if not args:
            return self._sro
        rmap = self._data.species_rmap
        fwd = self._data.species_map

        def z_of(x):
            return SYMBOL_MAP[x] if isinstance(x, str) else int(x)

        def one(shell, i, j):
            if shell not in self._data.shell_map:
                raise ValueError(f"This result does not contain a shell {shell}")
            zi, zj = z_of(i), z_of(j)
            if zi not in fwd or zj not in fwd:
                raise ValueError("This result does not contain the requested species")
            return SroParameter(shell, zi, zj, self._sro[self._data.shell_map[shell], fwd[zi], fwd[zj]])

        if len(args) == 3:
            return one(*args)
        if len(args) == 1:
            zs = [rmap[k] for k in sorted(rmap)]
            return [one(args[0], zs[a], zs[b]) for a in range(len(zs)) for b in range(a, len(zs))]
        if len(args) == 2:
            return [one(s, args[0], args[1]) for s in sorted(self._data.shell_map)]
        raise TypeError("sro() takes 0, 1, 2 or 3 arguments")

    def structure(self) -> Structure:
        return self._data.structure.with_species(self.species)

    def rank(self) -> str:
        """1-based rank of the configuration over all its species (results.h:156-162)."""
        packed = np.array([self._data.species_map[z] for z in self.species], dtype=np.uint8)
        return str(_native.rank_permutation(packed))

    def shell_index(self, shell):
        return self._data.shell_map.get(shell)

    def species_index(self, z):
        return self._data.species_map.get(z)

    def __repr__(self) -> str:
        return f"SqsResult(objective={self.objective!r})"


class SqsResultSplit:
    """A split-mode result: total objective plus one interact result per sublattice."""

    def __init__(self, objective, sublattices: list[SqsResult], base: Structure, site_lists):
        self.objective = objective
        self.sublattices = sublattices
        self._base = base
        self._sites = site_lists

    @property
    def species(self) -> list[int]:
        sp = list(self._base.species)
        for sl, sites in zip(self.sublattices, self._sites):
            for k, i in enumerate(sites):
                sp[i] = sl.species[k]
        return sp

    def structure(self) -> Structure:
        return self._base.with_species(self.species)

    def __repr__(self) -> str:
        return f"SqsResultSplit(objective={self.objective!r})"


@dataclass
class SroParameter:
    shell: int
    i: int
    j: int
    value: float


class SqsResultPack:
    """Results grouped by objective, ascending (``sqs_result_pack``, core/results.h:336-389)."""

    def __init__(self, config: SqsConfiguration, results, statistics: SqsStatistics):
        self.config = config
        self.statistics = statistics
        groups: dict = {}
        for r in results:
            groups.setdefault(r.objective, []).append(r)
        self.results = sorted(groups.items(), key=lambda kv: kv[0])

    def __iter__(self):
        return iter(self.results)

    def __len__(self) -> int:
        return len(self.results)

    def __getitem__(self, index):
        return self.results[index]

    def num_objectives(self) -> int:
        return len(self.results)

    def num_results(self) -> int:
        return sum(len(v) for _, v in self.results)

    def bytes(self) -> bytes:
        """The msgpack document of the pack (``pack.bytes()`` of the reference, io/json.h:264-275)."""
        from .io import dump_result_pack

        return dump_result_pack(self)

    @staticmethod
    def from_bytes(data: bytes, prec: Prec = Prec.single) -> "SqsResultPack":
        from .io import load_result_pack

        return load_result_pack(data, prec)

    def best(self):
        if not self.results:
            raise IndexError("No results available")
        return self.results[0][1][0]
