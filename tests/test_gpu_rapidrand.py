"""Reference-stream debug mode (option "rapidrand"): random jobs follow the reference's seeded
single-thread run instead of this library's stream. Its words come from rapidrand (core/shuffle.h:23-32);
the work is split into thread-pool blocks of chunk_size configurations (sqs.h:461-466) that restart
from the packed arrangement (sqs.h:374) while the stream continues; interact mode evaluates and then
shuffles (sqs.h:397-403,439-440), split mode shuffles every sublattice and then evaluates
(sqs.h:404-413). The device trace must equal that trajectory, restated here with the oracle's rapidrand
shuffle, configuration by configuration, with bit-exact bonds and objective; and the result set must
equal the deterministic core of the oracle's single-thread run (include/sqsgen/core/results.h:42-99)."""

import ctypes as C
import math

import numpy as np
import pytest

import cases
import oracle
import sqsgenerator_b200 as S
from sqsgenerator_b200 import _native as N
from sqsgenerator_b200.optimize import build_job

pytestmark = pytest.mark.gpu

# name -> (config, sublattice mode)
CASES = {
    "fcc32_interact_double": lambda: (cases.fcc32("double", iterations=6001, chunk_size=1500, seed=123, keep=4,
                                                  pair_weights=None), "interact"),
    "quinary108_interact_single": lambda: (cases.quinary("single", iterations=3001, chunk_size=700, seed=5, keep=3),
                                           "interact"),
    "rocksalt_split_double": lambda: (cases.rocksalt_split("double", iterations=3000, chunk_size=1000, seed=9, keep=3),
                                      "split"),
}


def _blocks(n, chunk):
    """The thread-pool blocks of [0, n) for one thread (BS_thread_pool v5, sqs.h:461-466)."""
    nb = n // chunk if chunk else 0
    nb = max(1, min(max(nb, 1), n))
    bs, rem = n // nb, n % nb
    starts = [b * bs + min(b, rem) for b in range(nb)]
    return list(zip(starts, starts[1:] + [n]))


def _trajectory(d, n, chunk, seed, split):
    """Every configuration of the reference's seeded single-thread run, in iteration order."""
    seeds = [seed] * len(d)  # one seed copied to every sublattice (io/config/combined.h:62-65)
    out = []
    for first, last in _blocks(n, chunk):
        cur = [x.species_packed.astype(np.uint8).copy() for x in d]
        for _ in range(first, last):
            if split:
                for p in range(len(d)):
                    cur[p], seeds[p] = oracle.shuffle_random(cur[p], d[p].windows, seeds[p])
                out.append(np.concatenate(cur))
            else:
                out.append(cur[0].copy())
                cur[0], seeds[0] = oracle.shuffle_random(cur[0], d[0].windows, seeds[0])
    return np.array(out, dtype=np.uint8)


@pytest.mark.parametrize("name", sorted(CASES))
def test_rapidrand_trace_is_the_reference_trajectory(name):
    cfg, mode = CASES[name]()
    n = cfg["iterations"]
    with N.options(rapidrand=1):
        c, d, _, sp, bd, ob, ids = cases.trace(cfg, n)
    assert len(ob) == n
    assert np.array_equal(ids, np.arange(n, dtype=np.uint64))  # ids are the reference's iteration indices
    want = _trajectory(d, n, int(c.chunk_size), int(cfg["seed"]), mode == "split")
    assert sp.shape == want.shape
    bad = np.nonzero((sp != want).any(axis=1))[0]
    assert len(bad) == 0, f"first differing iteration {bad[:5]}"
    assert cases.trace_mismatches(d, sp, bd, ob, cfg["prec"]) == []


@pytest.mark.parametrize("name", sorted(CASES))
def test_rapidrand_result_set_equals_single_thread_oracle(name):
    cfg, mode = CASES[name]()
    n = cfg["iterations"]
    c = S.parse_config(cfg)
    d = S.prepare(c)
    job, keep_alive = build_job(c, d)
    with N.options(rapidrand=1):
        plan = N.plan(job)
        assert [x["path"] for x in plan["parts"]] == ["general"] * len(d)
        run = C.c_void_p()
        N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
    L = N.lib()
    try:
        m = int(L.sqsg_run_count(run))
        T = np.float64 if cfg["prec"] == "double" else np.float32
        nsp = sum(len(x.species_packed) for x in d)
        nsro = sum(x.prefactors.size for x in d)
        obj = np.zeros(max(m, 1), T)
        sp = np.zeros(max(m, 1) * nsp, np.uint8)
        sro = np.zeros(max(m, 1) * nsro, T)
        ids = np.zeros(max(m, 1), np.uint64)
        N.check(L.sqsg_run_copy(run, 0, m, N.ptr(obj), None, N.ptr(sp), N.ptr(sro), N.ptr(ids)))
        st = N.SqsgStatistics()
        N.check(L.sqsg_run_statistics(run, C.byref(st)))
        assert int(st.finished) == n
    finally:
        L.sqsg_run_free(run)
    gpu = {(sp[k * nsp:(k + 1) * nsp].tobytes(), obj[k].tobytes(), sro[k * nsro:(k + 1) * nsro].tobytes())
           for k in range(m)}
    assert len(gpu) == m
    res, _ = oracle.optimize(d, prec=cfg["prec"], iteration_mode="random", sublattice_mode=mode, iterations=n,
                             chunk_size=int(c.chunk_size), keep=int(c.keep), threads=1,
                             seeds=[int(cfg["seed"])] * len(d))
    objs = sorted({float(r["objective"]) for r in res})
    tstar = objs[int(c.keep)] if len(objs) > int(c.keep) else math.inf
    core = {(np.concatenate(r["species"]).tobytes(), T(r["objective"]).tobytes(),
             np.concatenate([x.reshape(-1) for x in r["sro"]]).astype(T).tobytes())
            for r in res if float(r["objective"]) <= tstar}
    assert gpu == core


def test_rapidrand_is_refused_by_the_server_and_for_ranges():
    cfg, _ = CASES["fcc32_interact_double"]()
    c = S.parse_config(cfg)
    d = S.prepare(c)
    job, keep_alive = build_job(c, d)
    job.range_first, job.range_count = 10, 100
    with N.options(rapidrand=1):
        run = C.c_void_p()
        with pytest.raises(N.NativeError) as e:
            N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
        assert e.value.status_name == "SQSG_ERR_UNSUPPORTED"
        srv = S.Server(0)
        try:
            with pytest.raises(N.NativeError):
                srv.wait_run(srv.submit(None, prepared=(c, d)), timeout=60)
        finally:
            srv.close()
