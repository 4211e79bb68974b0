"""``optimize``: the drop-in for the reference's ``sqsgenerator.optimize``.

``prepare`` restates ``optimization_config::from_config`` (include/sqsgen/core/optimization_config.h:59-141):
sort sites by sublattice, pack species to dense indices, build the pair list of the sorted structure and
scale the pair weights by the shell weights. ``optimize`` hands the flattened job to the native engine
through the C ABI (``sqsg_optimize``) and maps the packed results back to atomic numbers in the original
site order like ``postprocess_results`` (include/sqsgen/sqs.h:95-122).
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Callable

import numpy as np

from . import _native
from .config import parse_config
from .core import (IterationMode, LogLevel, OptimizationData, ParseError, SqsConfiguration, SqsResult,
                   SqsResultPack, SqsResultSplit, SqsStatistics, Structure, SublatticeMode, dtype_of)

TIMING_NAMES = ("total", "chunk_setup", "loop", "comm")


def _scaled_pair_weights(pw, weights, K, T):
    """core/optimization.h:17-33."""
    w = np.array(pw, dtype=T, copy=True)
    for s, shell in enumerate(sorted(weights)):
        ws = T(weights[shell])
        for xi in range(K):
            for eta in range(xi, K):
                w[s, xi, eta] = T(w[s, xi, eta] * ws)
                if xi != eta:
                    w[s, eta, xi] = T(w[s, eta, xi] * ws)
    return w


def _index_mapping(values):
    zs = sorted(set(int(v) for v in values))
    return {z: i for i, z in enumerate(zs)}, {i: z for i, z in enumerate(zs)}


def prepare(config: SqsConfiguration) -> list[OptimizationData]:
    """Per-(sub)lattice optimisation data for a parsed configuration."""
    T = dtype_of(config.prec)
    structure = config.structure()
    from .config import apply_composition

    applied = structure.with_species(apply_composition(structure.species, config.composition))
    out = []
    if config.sublattice_mode == SublatticeMode.interact:
        n = len(applied)
        sl_of = np.full(n, len(config.composition), dtype=np.uint32)
        for k, sl in enumerate(config.composition):
            sl_of[np.asarray(sl.sites, dtype=np.int64)] = k
        order, windows = _native.sort_by_sublattice(sl_of, len(config.composition))
        # windows cover the sublattices only (sites in no sublattice sort last and are never shuffled)
        windows = windows[: len(config.composition)]
        sorted_struct = Structure(applied.lattice.copy(), applied.frac_coords[order].copy(),
                                  [applied.species[i] for i in order])
        parts = [(applied, sorted_struct, order, windows, config.composition)]
    else:
        parts = []
        for sl in config.composition:
            st = applied.sliced(sl.sites)
            parts.append((st, st, np.arange(len(st), dtype=np.uint32),
                          np.array([[0, len(st)]], dtype=np.uint32), [sl]))
    # supercell hint: supercell site k of a x b x c copies of n0 unit-cell sites is
    # k = ((i * b + j) * c + l) * n0 + s (the supercell loop order, core/structure.h:335-366)
    a, b, c = (int(v) for v in config.supercell)
    n0 = len(config.structure_config)

    def supercell_coords(indices):
        idx = np.asarray(indices, dtype=np.int64)
        s_, cell = idx % n0, idx // n0
        l_ = cell % c
        j_ = (cell // c) % b
        i_ = cell // (b * c)
        _, basis = np.unique(s_, return_inverse=True)
        return np.stack([basis, i_, j_, l_], axis=1).astype(np.uint32)

    hints = []
    if config.sublattice_mode == SublatticeMode.interact:
        hints.append(supercell_coords(parts[0][2]))
    else:
        for sl in config.composition:
            hints.append(supercell_coords(sl.sites))
    for k, (st, sst, order, windows, sls) in enumerate(parts):
        radii = config.shell_radii[k]
        weights = config.shell_weights[k]
        fwd, rev = _index_mapping(sst.species)
        packed = np.array([fwd[z] for z in sst.species], dtype=np.uint8)
        sm = sst.shell_matrix(radii)
        pairs = _native.pairs(sm, list(weights.keys()))
        K = len(fwd)
        shell_map = {s: i for i, s in enumerate(sorted(weights))}
        out.append(OptimizationData(
            structure=st, sorted_structure=sst, sort_order=np.asarray(order, dtype=np.int64),
            windows=np.asarray(windows, dtype=np.uint32), species_packed=packed, species_map=fwd,
            species_rmap=rev, shell_map=shell_map, pairs=pairs,
            prefactors=np.ascontiguousarray(config.prefactors[k], dtype=T),
            pair_weights=_scaled_pair_weights(config.pair_weights[k], weights, K, T),
            target=np.ascontiguousarray(config.target_objective[k], dtype=T),
            shell_radii=np.asarray(radii), shell_weights=dict(weights), sublattices=sls,
            lattice=hints[k], cells=(a, b, c)))
    return out


class _JobBuffers:
    """Keeps the numpy arrays that a native job points into alive."""

    def __init__(self):
        self.keep = []

    def add(self, a):
        a = np.ascontiguousarray(a)
        self.keep.append(a)
        return _native.ptr(a)


def build_job(config: SqsConfiguration, data: list[OptimizationData], device: int = 0,
              callback=None, cancel=None, lattice_hint: bool = True):
    """The flat ``sqsg_job`` for a configuration (C ABI struct + buffers to keep alive). With
    ``lattice_hint`` the supercell coordinates of the sites are passed on (the library checks them and
    may count bonds with translated bit planes; the result is the same either way)."""
    bufs = _JobBuffers()
    T = dtype_of(config.prec)
    subs = (_native.SqsgSublattice * len(data))()
    for k, d in enumerate(data):
        s = subs[k]
        s.n_sites = len(d.species_packed)
        s.n_species = d.prefactors.shape[1]
        s.n_shells = d.prefactors.shape[0]
        s.n_pairs = len(d.pairs)
        s.n_windows = len(d.windows)
        s.pairs = bufs.add(np.asarray(d.pairs, dtype=np.uint32).reshape(-1))
        s.species = bufs.add(d.species_packed.astype(np.uint8))
        s.windows = bufs.add(np.asarray(d.windows, dtype=np.uint32).reshape(-1))
        s.prefactors = bufs.add(d.prefactors.astype(T))
        s.pair_weights = bufs.add(d.pair_weights.astype(T))
        s.target = bufs.add(d.target.astype(T))
        if lattice_hint and d.lattice is not None:
            s.lattice = bufs.add(np.ascontiguousarray(d.lattice, dtype=np.uint32).reshape(-1))
            s.cells[0], s.cells[1], s.cells[2] = (int(v) for v in d.cells)
            s.n_basis = int(d.lattice[:, 0].max()) + 1
    bufs.keep.append(subs)
    job = _native.SqsgJob()
    job.prec = int(config.prec)
    job.iteration_mode = int(config.iteration_mode)
    job.sublattice_mode = int(config.sublattice_mode)
    job.n_sublattices = len(data)
    job.sublattices = C.cast(subs, C.c_void_p)
    job.iterations = 0 if config.iteration_mode == IterationMode.systematic else int(config.iterations)
    job.chunk_size = int(config.chunk_size)
    job.keep = int(config.keep)
    job.max_results_per_objective = -1 if config.max_results_per_objective is None else int(
        config.max_results_per_objective)
    seeds = [s for s in config.seed if s is not None]
    job.has_seed = 1 if seeds else 0
    job.seed = int(seeds[0]) & ((1 << 64) - 1) if seeds else 0
    job.device = device
    if cancel is not None:
        job.cancel = C.cast(cancel, C.c_void_p)
    if callback is not None:
        job.callback = callback
        bufs.keep.append(callback)
    return job, bufs


def collect(config: SqsConfiguration, data: list[OptimizationData], run) -> SqsResultPack:
    """Turn a native run handle into an ``SqsResultPack`` (packed -> Z, sorted -> original order)."""
    L = _native.lib()
    T = dtype_of(config.prec)
    n = int(L.sqsg_run_count(run))
    nsl = len(data)
    sizes = [(len(d.species_packed), d.prefactors.shape[0], d.prefactors.shape[1]) for d in data]
    tot_sp = sum(x[0] for x in sizes)
    tot_sro = sum(x[1] * x[2] * x[2] for x in sizes)
    obj = np.zeros(max(n, 1), dtype=T)
    sub = np.zeros(max(n, 1) * nsl, dtype=T)
    sp = np.zeros(max(n, 1) * tot_sp, dtype=np.uint8)
    sro = np.zeros(max(n, 1) * tot_sro, dtype=T)
    ids = np.zeros(max(n, 1), dtype=np.uint64)
    if n:
        _native.check(L.sqsg_run_copy(run, 0, n, _native.ptr(obj), _native.ptr(sub), _native.ptr(sp),
                                      _native.ptr(sro), _native.ptr(ids)))
    st = _native.SqsgStatistics()
    _native.check(L.sqsg_run_statistics(run, C.byref(st)))
    stats = SqsStatistics(int(st.finished), int(st.working), int(st.best_rank), float(st.best_objective),
                          {name: int(st.timings_ns[i]) for i, name in enumerate(TIMING_NAMES)})
    sp = sp.reshape(max(n, 1), tot_sp)
    sro = sro.reshape(max(n, 1), tot_sro)
    sub = sub.reshape(max(n, 1), nsl)
    results = []
    for r in range(n):
        o1 = o2 = 0
        per = []
        for k, (d, (N, S, K)) in enumerate(zip(data, sizes)):
            packed = sp[r, o1:o1 + N]
            cube = sro[r, o2:o2 + S * K * K].reshape(S, K, K).copy()
            z = np.array([d.species_rmap[int(x)] for x in packed], dtype=np.int64)
            original = np.empty(N, dtype=np.int64)
            original[d.sort_order] = z
            per.append(SqsResult(T(sub[r, k]), original.tolist(), cube, d, int(ids[r])))
            o1 += N
            o2 += S * K * K
        if config.sublattice_mode == SublatticeMode.interact:
            res = per[0]
            res.objective = T(obj[r])
            results.append(res)
        else:
            base = data[0].structure
            full = config.structure()
            from .config import apply_composition
            full = full.with_species(apply_composition(full.species, config.composition))
            results.append(SqsResultSplit(T(obj[r]), per, full, [sl.sites for sl in config.composition]))
            del base
    return SqsResultPack(config, results, stats)


def optimize(config: dict[str, Any] | SqsConfiguration | str, level: LogLevel = LogLevel.warn,
             callback: Callable | None = None, device: int = 0) -> SqsResultPack:
    """Run the optimisation on one GPU and return the reference-shaped result pack.

    ``callback(statistics)`` is called from this thread while the device works; returning a truthy
    value (or calling ``.stop()`` on the passed context) stops the run early.
    """
    c = config if isinstance(config, SqsConfiguration) else parse_config(config)
    if isinstance(c, ParseError):
        raise ValueError(str(c))
    data = prepare(c)
    cb = None
    if callback is not None:
        def _cb(stats_ptr, user):
            s = stats_ptr.contents
            ctx = _CallbackContext(SqsStatistics(int(s.finished), int(s.working), int(s.best_rank),
                                                 float(s.best_objective),
                                                 {n: int(s.timings_ns[i]) for i, n in enumerate(TIMING_NAMES)}))
            try:
                ret = callback(ctx)
            except Exception:  # noqa: BLE001 — a failing callback stops the run
                return 1
            return 1 if (ret or ctx.stopped) else 0
        cb = _native.CALLBACK(_cb)
    job, bufs = build_job(c, data, device=device, callback=cb)
    run = C.c_void_p()
    _native.check(_native.lib().sqsg_optimize(C.byref(job), C.byref(run)))
    try:
        return collect(c, data, run)
    finally:
        _native.lib().sqsg_run_free(run)


class _CallbackContext:
    """``sqs_callback_context`` (include/sqsgen/types.h:222-235)."""

    def __init__(self, statistics: SqsStatistics):
        self.statistics = statistics
        self.stopped = False

    def stop(self) -> None:
        self.stopped = True
