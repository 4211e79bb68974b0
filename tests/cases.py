"""Configurations shared by the tests (reference-schema dicts) and trace helpers."""
from __future__ import annotations

import ctypes as C

import numpy as np

import oracle
from oracle import geometry as G


def fcc_coords():
    return [[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]


def settings_16(prec="double"):
    """python/tests/test_core.py:28-44 of the reference: a 16-site cell, Ti8Al8 on the H sites."""
    return dict(
        prec=prec,
        iteration_mode="systematic",
        structure=dict(lattice=np.diag([1, 2, 3]).tolist(),
                       coords=[[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5]],
                       species=[1] * 4, supercell=[2, 2, 1]),
        pair_weights=0,
        composition={"sites": "H", "Ti": 8, "Al": 8},
        thread_config=1,
    )


def fcc32(prec="double", **kw):
    """fcc 2x2x2 (32 sites, a = 4.0), A16B16, shells 1/2 weighted 1.0/0.5, all pair weights 1."""
    a = 4.0
    d = dict(prec=prec,
             structure=dict(lattice=(np.eye(3) * a).tolist(), coords=fcc_coords(), species=[1] * 4, supercell=[2, 2, 2]),
             composition={"Ti": 16, "Al": 16}, shell_weights={"1": 1.0, "2": 0.5}, pair_weights=1,
             iterations=1000000, seed=42, thread_config=1, keep=10)
    d.update(kw)
    return {k: v for k, v in d.items() if v is not None}


def quinary(prec="double", cells=(3, 3, 3), **kw):
    a = 4.0
    n = 4 * cells[0] * cells[1] * cells[2]
    counts = [n // 5 + (1 if k < n % 5 else 0) for k in range(5)]
    comp = dict(zip(["Ti", "Al", "Nb", "V", "Zr"], counts))
    d = dict(prec=prec,
             structure=dict(lattice=(np.eye(3) * a).tolist(), coords=fcc_coords(), species=[1] * 4, supercell=list(cells)),
             composition=comp, shell_weights={"1": 1.0, "2": 0.5, "3": 0.25}, iterations=20000, seed=7,
             thread_config=1, keep=5)
    d.update(kw)
    return d


def rocksalt_split(prec="double", cells=(2, 2, 2), **kw):
    L, F = G.rocksalt(4.2)
    n = 4 * cells[0] * cells[1] * cells[2]
    d = dict(prec=prec, sublattice_mode="split",
             structure=dict(lattice=L.tolist(), coords=F.tolist(), species=[11] * 4 + [17] * 4, supercell=list(cells)),
             composition=[{"sites": "Na", "Ti": n // 2, "Al": n - n // 2},
                          {"sites": "Cl", "N": n - n // 8, "B": n // 8}],
             shell_weights=[{"1": 1.0, "2": 0.5}, {"1": 1.0, "2": 0.5}], iterations=20000, seed=3, thread_config=1)
    d.update(kw)
    return d


def trace(config, capacity):
    """Run through sqsg_optimize_trace; returns (config, data, pack, species, bonds, objective, ids)."""
    import sqsgenerator_b200 as S
    from sqsgenerator_b200 import _native as N
    from sqsgenerator_b200.optimize import build_job, collect

    c = S.parse_config(config)
    assert not isinstance(c, S.ParseError), c
    d = S.prepare(c)
    job, bufs = build_job(c, d)
    T = np.float64 if int(c.prec) == 1 else np.float32
    sp_w = sum(len(x.species_packed) for x in d)
    bd_w = sum(x.prefactors.size for x in d)
    sp = np.zeros(capacity * sp_w, np.uint8)
    bd = np.zeros(capacity * bd_w, np.uint32)
    ob = np.zeros(capacity, T)
    ids = np.zeros(capacity, np.uint64)
    cnt = C.c_uint64(0)
    run = C.c_void_p()
    N.check(N.lib().sqsg_optimize_trace(C.byref(job), C.byref(run), capacity, C.byref(cnt), N.ptr(sp), N.ptr(bd),
                                        N.ptr(ob), N.ptr(ids)))
    try:
        pack = collect(c, d, run)
    finally:
        N.lib().sqsg_run_free(run)
    n = min(cnt.value, capacity)
    return c, d, pack, sp[: n * sp_w].reshape(n, sp_w), bd[: n * bd_w].reshape(n, bd_w), ob[:n], ids[:n]


def trace_mismatches(d, sp, bd, ob, prec, limit=None):
    """Recompute ordered bonds and objective of every traced configuration with the oracle, and check
    that each is an arrangement of the packed one (every window keeps its species multiset, sites outside
    the windows keep theirs); return the mismatching rows."""
    n = len(ob) if limit is None else min(limit, len(ob))
    T = np.float64 if prec in ("double", 1) else np.float32
    bad = []
    total = None
    bonds_ok = np.ones(n, dtype=bool)
    comp_ok = np.ones(n, dtype=bool)
    o1 = o2 = 0
    for part in d:
        npart = len(part.species_packed)
        skk = part.prefactors.size
        rows = sp[:n, o1:o1 + npart]
        packed = np.asarray(part.species_packed)
        fixed = np.ones(npart, dtype=bool)
        for lo, hi in np.asarray(part.windows).tolist():
            fixed[lo:hi] = False
            comp_ok &= np.all(np.sort(rows[:, lo:hi], axis=1) == np.sort(packed[lo:hi]), axis=1)
        comp_ok &= np.all(rows[:, fixed] == packed[fixed], axis=1)
        b, o = oracle.evaluate_many(part, rows, prec)
        bonds_ok &= np.all(b.reshape(n, skk).astype(np.uint32) == bd[:n, o2:o2 + skk], axis=1)
        total = o if total is None else (total + o).astype(T)
        o1 += npart
        o2 += skk
    obj_ok = total.view(np.uint32 if T is np.float32 else np.uint64) == np.asarray(ob[:n], T).view(
        np.uint32 if T is np.float32 else np.uint64)
    for k in np.flatnonzero(~(bonds_ok & obj_ok & comp_ok))[:20]:
        what = "composition" if not comp_ok[k] else ("bonds" if not bonds_ok[k] else "objective")
        bad.append((int(k), what, total[k], ob[k]))
    return bad


def run_levels(run):
    """(values, counts, checksums) of a native run handle."""
    from sqsgenerator_b200 import _native as N

    cap = 1100  # keep <= 1023: up to 1024 levels
    n = C.c_uint32(cap)
    v = np.zeros(cap, np.float64)
    cnt = np.zeros(cap, np.uint64)
    cs = np.zeros(cap, np.uint64)
    N.check(N.lib().sqsg_run_levels(run, C.byref(n), N.ptr(v), N.ptr(cnt), N.ptr(cs)))
    return [(float(v[i]), int(cnt[i]), int(cs[i])) for i in range(n.value)]


def oracle_fcc32(T=np.float64):
    """The fcc 2x2x2 A16B16 benchmark cell built by the oracle's own geometry (independent of the
    product's precompute): shells 1/2 weighted 1.0/0.5, all pair weights 1."""
    lat, frac = G.fcc(4.0)
    L, F, species = G.supercell(lat, frac, [1] * 4, 2, 2, 2, T)
    comp = [(set(range(32)), {13: 16, 22: 16})]
    radii = G.distances_histogram(G.distance_matrix(L, F, T), 0.05, 0.25, T)
    return G.prepare_interact(L, F, species, comp, radii, {1: T(1.0), 2: T(0.5)}, T,
                              pair_weights=np.ones((2, 2, 2), dtype=T))
