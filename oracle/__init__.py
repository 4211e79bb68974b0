"""Oracle for the SQS optimisation hot path — TEST INFRASTRUCTURE ONLY.

The oracle is a CPU restatement of the reference (dgehringer/sqsgenerator 0.5.6) path that the GPU
product replaces: ``liboracle.so`` (C++, ``oracle/sqsg_oracle.cpp``) restates the optimizer loop,
``count_bonds``, ``compute_objective``, the rapidrand shuffler, multiset permutation (un)ranking and
the result collection; ``oracle/geometry.py`` restates the host-side geometry precompute.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its ``cpu_baseline`` leg and its
``--impl reference`` arm) may import this package, and only as the checker or the timed CPU baseline.
The product package ``sqsgenerator_b200`` never imports it.

Pinning: the permutation functions, the geometry (distance matrix, shell matrix, naive radii,
supercell, prefactors) and the bond/SRO relation are checked against the reference's own test
vectors (``tests/golden``, generated from the reference's tests by ``tests/golden/make_golden.py``).
The objective value and the rapidrand sequence have no golden numbers in the reference; they are
pinned by restating ``core/optimization.h:79-103`` and ``core/shuffle.h:23-32`` operation for
operation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class Sublattice(C.Structure):
    _fields_ = [
        ("n_sites", C.c_int32),
        ("n_species", C.c_int32),
        ("n_shells", C.c_int32),
        ("n_pairs", C.c_int32),
        ("n_bounds", C.c_int32),
        ("has_seed", C.c_int32),
        ("pairs", C.c_void_p),
        ("species_packed", C.c_void_p),
        ("bounds", C.c_void_p),
        ("prefactors", C.c_void_p),
        ("pair_weights", C.c_void_p),
        ("target", C.c_void_p),
        ("seed", C.c_uint64),
    ]


class Job(C.Structure):
    _fields_ = [
        ("prec", C.c_int32),
        ("iteration_mode", C.c_int32),
        ("sublattice_mode", C.c_int32),
        ("n_sublattices", C.c_int32),
        ("sublattices", C.c_void_p),
        ("iterations", C.c_uint64),
        ("chunk_size", C.c_uint64),
        ("keep", C.c_uint64),
        ("max_results_per_objective", C.c_int64),
        ("threads", C.c_int32),
        ("share_seed_across_threads", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("finished", C.c_uint64),
        ("best_rank", C.c_uint64),
        ("best_objective", C.c_double),
        ("seconds", C.c_double),
    ]


def lib():
    """Load (building on first use when sources are present) ``oracle/liboracle.so``."""
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path) or (
            os.path.exists(_build.SRC) and os.path.getmtime(path) < os.path.getmtime(_build.SRC)
        ):
            _build.build()
        L = C.CDLL(path)
        L.oracle_rapidrand.restype = C.c_uint64
        L.oracle_rapidrand.argtypes = [C.POINTER(C.c_uint64)]
        L.oracle_random_bounded.restype = C.c_uint64
        L.oracle_random_bounded.argtypes = [C.c_uint64, C.POINTER(C.c_uint64)]
        L.oracle_shuffle_random.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_uint64)]
        L.oracle_num_permutations.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_uint64)]
        L.oracle_rank_permutation.restype = C.c_uint64
        L.oracle_rank_permutation.argtypes = [C.c_void_p, C.c_int]
        L.oracle_unrank_permutation.argtypes = [C.c_void_p, C.c_int, C.c_uint64]
        L.oracle_next_permutation.argtypes = [C.c_void_p, C.c_int]
        L.oracle_count_bonds.argtypes = [C.POINTER(Sublattice), C.c_void_p, C.c_void_p]
        L.oracle_evaluate_d.restype = C.c_double
        L.oracle_evaluate_d.argtypes = [C.POINTER(Sublattice), C.c_void_p, C.c_void_p]
        L.oracle_evaluate_f.restype = C.c_float
        L.oracle_evaluate_f.argtypes = [C.POINTER(Sublattice), C.c_void_p, C.c_void_p]
        L.oracle_evaluate_many.argtypes = [C.POINTER(Sublattice), C.c_int, C.c_uint64, C.c_void_p, C.c_void_p,
                                           C.c_void_p]
        L.oracle_optimize.restype = C.c_void_p
        L.oracle_optimize.argtypes = [C.POINTER(Job)]
        L.oracle_result_free.argtypes = [C.c_void_p]
        L.oracle_result_count.restype = C.c_uint64
        L.oracle_result_count.argtypes = [C.c_void_p]
        L.oracle_result_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.oracle_result_get.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_sort_by_sublattice.restype = C.c_int
        L.oracle_sort_by_sublattice.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_systematic_levels.restype = C.c_int
        L.oracle_systematic_levels.argtypes = [C.POINTER(Sublattice), C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                               C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        _LIB = L
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


# ----------------------------------------------------------------------------- permutations / rng
def rapidrand(seed: int):
    s = C.c_uint64(seed)
    v = lib().oracle_rapidrand(C.byref(s))
    return int(v), int(s.value)


def shuffle_random(species, bounds, seed: int):
    c = np.ascontiguousarray(species, dtype=np.uint8).copy()
    b = np.ascontiguousarray(bounds, dtype=np.uint32).reshape(-1)
    s = C.c_uint64(seed)
    lib().oracle_shuffle_random(_ptr(c), _ptr(b), len(b) // 2, C.byref(s))
    return c, int(s.value)


def num_permutations(conf):
    c = np.ascontiguousarray(conf, dtype=np.uint8)
    out = C.c_uint64(0)
    ok = lib().oracle_num_permutations(_ptr(c), len(c), C.byref(out))
    return int(out.value) if ok else None


def rank_permutation(conf):
    c = np.ascontiguousarray(conf, dtype=np.uint8)
    return int(lib().oracle_rank_permutation(_ptr(c), len(c)))


def unrank_permutation(conf, rank):
    c = np.ascontiguousarray(conf, dtype=np.uint8).copy()
    if not lib().oracle_unrank_permutation(_ptr(c), len(c), rank):
        raise IndexError("The rank is larger than the total number of permutations")
    return c


def next_permutation(conf):
    c = np.ascontiguousarray(conf, dtype=np.uint8).copy()
    ok = lib().oracle_next_permutation(_ptr(c), len(c))
    return c, bool(ok)


# ----------------------------------------------------------------------------- sublattice packing
class _Keep:
    """Keeps the numpy buffers a ctypes struct points into alive."""

    def __init__(self):
        self.bufs = []

    def add(self, a):
        self.bufs.append(a)
        return _ptr(a)


def make_sublattice(sd, prec_dtype, seed=None, keep=None):
    """ctypes struct for a ``geometry.SublatticeData``-like object (attributes species_packed, pairs,
    bounds or windows, prefactors, pair_weights, target)."""
    keep = keep if keep is not None else _Keep()
    T = np.float64 if prec_dtype in (np.float64, "double", 1) else np.float32
    pairs = np.ascontiguousarray(sd.pairs, dtype=np.uint32).reshape(-1)
    sp = np.ascontiguousarray(sd.species_packed, dtype=np.uint8)
    bounds = np.ascontiguousarray(
        np.asarray(getattr(sd, "bounds", None) if hasattr(sd, "bounds") else sd.windows, dtype=np.uint32).reshape(-1))
    f = np.ascontiguousarray(sd.prefactors, dtype=T)
    w = np.ascontiguousarray(sd.pair_weights, dtype=T)
    t = np.ascontiguousarray(sd.target, dtype=T)
    S, K = f.shape[0], f.shape[1]
    s = Sublattice()
    s.n_sites = len(sp)
    s.n_species = K
    s.n_shells = S
    s.n_pairs = len(pairs) // 3
    s.n_bounds = len(bounds) // 2
    s.has_seed = 0 if seed is None else 1
    s.seed = 0 if seed is None else int(seed)
    s.pairs = keep.add(pairs)
    s.species_packed = keep.add(sp)
    s.bounds = keep.add(bounds)
    s.prefactors = keep.add(f)
    s.pair_weights = keep.add(w)
    s.target = keep.add(t)
    return s, keep


def count_bonds(sd, species):
    s, keep = make_sublattice(sd, np.float64)
    S, K = s.n_shells, s.n_species
    out = np.zeros(S * K * K, dtype=np.uint64)
    sp = np.ascontiguousarray(species, dtype=np.uint8)
    lib().oracle_count_bonds(C.byref(s), _ptr(sp), _ptr(out))
    return out.reshape(S, K, K)


def symmetrize_bonds(bonds):
    """Symmetrised counts n(s,a,b) = bonds(s,a,b) + bonds(s,b,a) off the diagonal."""
    b = np.asarray(bonds, dtype=np.int64)
    out = b + np.transpose(b, (0, 2, 1))
    for k in range(b.shape[1]):
        out[:, k, k] = b[:, k, k]
    return out


def evaluate(sd, species, prec="double"):
    """(objective, sro[S,K,K]) of one configuration, computed by the restated reference code."""
    T = np.float64 if prec in ("double", 1, np.float64) else np.float32
    s, keep = make_sublattice(sd, T)
    S, K = s.n_shells, s.n_species
    sro = np.zeros(S * K * K, dtype=T)
    sp = np.ascontiguousarray(species, dtype=np.uint8)
    if T is np.float64:
        o = lib().oracle_evaluate_d(C.byref(s), _ptr(sp), _ptr(sro))
    else:
        o = lib().oracle_evaluate_f(C.byref(s), _ptr(sp), _ptr(sro))
    return T(o), sro.reshape(S, K, K)


def evaluate_many(sd, species, prec="double"):
    """(bonds[n, S, K, K] ordered counts, objectives[n]) of many configurations at once."""
    T = np.float64 if prec in ("double", 1, np.float64) else np.float32
    s, keep = make_sublattice(sd, T)
    S, K = s.n_shells, s.n_species
    sp = np.ascontiguousarray(species, dtype=np.uint8)
    n = sp.shape[0]
    bonds = np.zeros((n, S * K * K), dtype=np.uint64)
    obj = np.zeros(n, dtype=T)
    lib().oracle_evaluate_many(C.byref(s), 1 if T is np.float64 else 0, n, _ptr(sp), _ptr(bonds), _ptr(obj))
    return bonds.reshape(n, S, K, K), obj


def optimize(sublattices, *, prec="double", iteration_mode="random", sublattice_mode="interact",
             iterations=100000, chunk_size=None, keep=1, max_results_per_objective=None,
             threads=1, seeds=None, share_seed=True):
    """Run the restated reference optimizer loop; returns (results, stats).

    ``results`` is a list of dicts sorted by objective then configuration: objective,
    sub_objectives, species (per sublattice, packed, sorted site order), sro (per sublattice,
    row-major [s][a][b]).
    """
    T = np.float64 if prec in ("double", 1, np.float64) else np.float32
    keepalive = _Keep()
    structs = (Sublattice * len(sublattices))()
    for k, sd in enumerate(sublattices):
        seed = None if seeds is None else seeds[k]
        s, _ = make_sublattice(sd, T, seed=seed, keep=keepalive)
        structs[k] = s
    if chunk_size is None:
        chunk_size = min(iterations, 100000)
    job = Job()
    job.prec = 1 if T is np.float64 else 0
    job.iteration_mode = 1 if iteration_mode == "systematic" else 0
    job.sublattice_mode = 1 if sublattice_mode == "split" else 0
    job.n_sublattices = len(sublattices)
    job.sublattices = C.cast(structs, C.c_void_p)
    job.iterations = int(iterations)
    job.chunk_size = int(chunk_size)
    job.keep = int(keep)
    job.max_results_per_objective = -1 if max_results_per_objective is None else int(max_results_per_objective)
    job.threads = int(threads)
    job.share_seed_across_threads = 1 if share_seed else 0
    L = lib()
    h = L.oracle_optimize(C.byref(job))
    if not h:
        raise RuntimeError(L.oracle_last_error().decode())
    try:
        n = L.oracle_result_count(h)
        st = Stats()
        L.oracle_result_stats(h, C.byref(st))
        sizes = [(s.n_sites, s.n_shells, s.n_species) for s in structs]
        tot_sites = sum(x[0] for x in sizes)
        tot_sro = sum(x[1] * x[2] * x[2] for x in sizes)
        out = []
        obj = np.zeros(1, dtype=T)
        sub = np.zeros(len(sizes), dtype=T)
        sp = np.zeros(tot_sites, dtype=np.uint8)
        sro = np.zeros(tot_sro, dtype=T)
        for i in range(n):
            L.oracle_result_get(h, i, _ptr(obj), _ptr(sub), _ptr(sp), _ptr(sro))
            species, sros = [], []
            o1 = o2 = 0
            for (ns, S, K) in sizes:
                species.append(sp[o1:o1 + ns].copy())
                sros.append(sro[o2:o2 + S * K * K].reshape(S, K, K).copy())
                o1 += ns
                o2 += S * K * K
            out.append(dict(objective=T(obj[0]), sub_objectives=sub.copy(), species=species, sro=sros))
        stats = dict(finished=st.finished, best_rank=st.best_rank, best_objective=st.best_objective,
                     seconds=st.seconds)
        return out, stats
    finally:
        L.oracle_result_free(h)


def systematic_levels(sd, *, prec="double", keep=1, threads=None, first=0, count=0):
    """Exhaustive enumeration of the single window (ranks first+1 .. first+count, all when count is
    0): the keep+1 best distinct objectives with their configuration counts and rank checksums
    (sums of the low / high halves of splitmix64(rank), mod 2^32).
    """
    T = np.float64 if prec in ("double", 1, np.float64) else np.float32
    s, keepalive = make_sublattice(sd, T)
    cap = int(keep) + 1
    vals = np.zeros(cap, dtype=np.float64)
    cnts = np.zeros(cap, dtype=np.uint64)
    sums = np.zeros(cap, dtype=np.uint64)
    n = lib().oracle_systematic_levels(C.byref(s), 1 if T is np.float64 else 0, int(threads or os.cpu_count() or 1),
                                       int(keep), int(first), int(count), _ptr(vals), _ptr(cnts), _ptr(sums), cap)
    if n < 0:
        raise RuntimeError(lib().oracle_last_error().decode())
    return [(float(vals[i]), int(cnts[i]), int(sums[i])) for i in range(n)]


def sort_by_sublattice(sl_of_site, n_sublattices):
    """(sort_order, windows) exactly as the reference's std::sort-based compute_shuffling_bounds."""
    s = np.ascontiguousarray(sl_of_site, dtype=np.uint32)
    n = len(s)
    order = np.zeros(n, dtype=np.uint32)
    cap = n_sublattices + 2
    win = np.zeros(2 * cap, dtype=np.uint32)
    k = lib().oracle_sort_by_sublattice(_ptr(s), n, int(n_sublattices), _ptr(order), _ptr(win), cap)
    return order.tolist(), [(int(win[2 * i]), int(win[2 * i + 1])) for i in range(k)]
