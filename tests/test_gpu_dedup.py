"""Random runs over small configuration spaces revisit the same configurations many times. When the
evaluations at or below the final (keep+1)-th best objective T* are too many for the re-run's record
budget, the re-run keeps each distinct configuration once, with its smallest id, in a device table
keyed by the exact configuration (the species bit mask on the bit-mask path, the multiset-permutation
rank elsewhere). The result set must still equal the rule restated here on a full trace of the run:
the keep+1 smallest distinct objectives, one record per distinct configuration (the smallest id),
ordered by objective then id — the reference's result collection (include/sqsgen/core/results.h:42-99)
— on the plain path and in the served form, for the bit-mask, general, lattice and split paths."""

import ctypes as C
import math

import numpy as np
import pytest

import cases
import sqsgenerator_b200 as S
from sqsgenerator_b200 import _native as N
from sqsgenerator_b200.optimize import build_job

pytestmark = pytest.mark.gpu


def _multinomial(counts):
    n, m = 0, 1
    for c in counts:
        n += c
        m *= math.comb(n, c)
    return m


# name -> (config, iterations, keep, options, arrangements of the species multisets)
CASES = {
    "bitmask_fcc32_a3b29": lambda: (
        cases.fcc32("double", composition={"Ti": 3, "Al": 29}, iterations=300000, seed=21, keep=4,
                    pair_weights=None), 300000, 4, {}, _multinomial([3, 29])),
    "general_fcc32_a3b29_single": lambda: (
        cases.fcc32("single", composition={"Ti": 3, "Al": 29}, iterations=300000, seed=22, keep=4,
                    pair_weights=None), 300000, 4, {"force_general": 1}, _multinomial([3, 29])),
    "lattice_fcc32_ternary": lambda: (
        cases.fcc32("double", composition={"Ti": 1, "Al": 30, "Nb": 1}, iterations=150000, seed=23, keep=3),
        150000, 3, {"use_tuning": 0}, _multinomial([1, 30, 1])),  # the rules' path: lattice
    "split_rocksalt": lambda: (
        cases.rocksalt_split("double", iterations=200000, seed=24, keep=3,
                             composition=[{"sites": "Na", "Ti": 1, "Al": 31}, {"sites": "Cl", "N": 31, "B": 1}]),
        200000, 3, {"use_tuning": 0}, _multinomial([1, 31]) * _multinomial([31, 1])),
}


PATH = {"bitmask_fcc32_a3b29": "bitmask", "general_fcc32_a3b29_single": "general", "lattice_fcc32_ternary": "lattice",
        "split_rocksalt": "lattice"}


def _expected(cfg, n, keep):
    """(expected records, evaluations at the keep+1 levels, distinct configurations at or below T*,
    levels) from a full trace of the run."""
    _, d, _, sp, _, ob, ids = cases.trace(cfg, n)
    assert len(ob) == n
    obl = ob.tolist()
    levels = sorted(set(obl))[: keep + 1]
    lset = set(levels)
    need = sum(1 for o in obl if o in lset)
    order = sorted((float(ob[k]), int(ids[k]), k) for k in range(n) if float(ob[k]) in lset)
    seen, expect = set(), []
    for o, i, k in order:
        key = sp[k].tobytes()
        if key in seen:
            continue
        seen.add(key)
        expect.append((o, i, key))
    return expect, need, len(seen), levels


def _records(run):
    L = N.lib()
    n = int(L.sqsg_run_count(run))
    nsp = _records.nsp
    obj = np.zeros(max(n, 1), np.float64 if _records.double else np.float32)
    sp = np.zeros(max(n, 1) * nsp, np.uint8)
    ids = np.zeros(max(n, 1), np.uint64)
    N.check(L.sqsg_run_copy(run, 0, n, N.ptr(obj), None, N.ptr(sp), None, N.ptr(ids)))
    cand, trunc, exact = C.c_uint64(), C.c_int32(), C.c_int32()
    N.check(L.sqsg_run_info(run, C.byref(cand), C.byref(trunc), C.byref(exact)))
    got = [(float(obj[k]), int(ids[k]), sp[k * nsp:(k + 1) * nsp].tobytes()) for k in range(n)]
    return got, dict(candidates=cand.value, truncated=bool(trunc.value), levels_exact=bool(exact.value))


@pytest.mark.parametrize("form", ["plain", "served"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_dedup_rerun_equals_full_trace(name, form):
    cfg, n, keep, opts, space = CASES[name]()
    expect, need, distinct, levels = _expected(cfg, n, keep)
    # the case must reach the deduplicating re-run: the evaluations at or below T* exceed the re-run
    # budget (set to `need` records), while the table for min(need, arrangements) fits in it
    bound = min(need, space)
    slots = 1024
    while slots < 2 * bound:
        slots *= 2
    assert bound + 64 + slots * 24 // 16 <= need, (need, bound, slots)
    assert distinct < need
    c = S.parse_config(cfg)
    d = S.prepare(c)
    _records.nsp = sum(len(x.species_packed) for x in d)
    _records.double = int(c.prec) == 1
    with N.options(**opts):
        job, bufs = build_job(c, d)
        plan = N.plan(job)
        assert plan["parts"][0]["path"] == PATH[name]
        record_bytes = plan["record_bytes"]
        with N.options(default_candidates=max(need // 4, 64), rerun_record_bytes=need * record_bytes):
            if form == "plain":
                run = C.c_void_p()
                N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
                try:
                    got, info = _records(run)
                    lv = cases.run_levels(run)
                finally:
                    N.lib().sqsg_run_free(run)
            else:
                srv = S.Server(0, default_max_results=max(need // 4, 64))
                try:
                    run = srv.wait_run(srv.submit(None, prepared=(c, d)), timeout=120)
                    try:
                        got, info = _records(run)
                        lv = cases.run_levels(run)
                    finally:
                        N.lib().sqsg_run_free(run)
                finally:
                    srv.close()
    assert not info["truncated"] and info["levels_exact"]
    assert info["candidates"] == distinct  # one candidate per distinct configuration: the table ran
    assert [v for v, _, _ in lv] == levels
    assert got == expect


def test_small_record_budget_truncates():
    """A random job whose re-run fits the record budget neither with every evaluation nor as a table of
    distinct configurations (C(32,16) arrangements: almost no repeats) keeps the first pass's records:
    the set is flagged truncated and the levels stay exact."""
    cfg = cases.fcc32("double", iterations=200000, seed=25, keep=4, pair_weights=None)
    c = S.parse_config(cfg)
    d = S.prepare(c)
    job, bufs = build_job(c, d)
    with N.options(default_candidates=1000, rerun_record_bytes=1000 * N.plan(job)["record_bytes"]):
        run = C.c_void_p()
        N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
    try:
        cand, trunc, exact = C.c_uint64(), C.c_int32(), C.c_int32()
        N.check(N.lib().sqsg_run_info(run, C.byref(cand), C.byref(trunc), C.byref(exact)))
        assert trunc.value == 1 and exact.value == 1
        assert int(N.lib().sqsg_run_count(run)) > 0
    finally:
        N.lib().sqsg_run_free(run)
