"""Batched and served forms: every job's result is the same alone (sqsg_optimize) and in the mix
(sqsg_optimize_batch, and the continuous-batching server with jobs arriving while others run)."""
import ctypes as C
import threading
import time

import numpy as np
import pytest

import cases
import sqsgenerator_b200 as S
from sqsgenerator_b200 import _native as N
from sqsgenerator_b200.optimize import build_job

pytestmark = pytest.mark.gpu


def _fcc555(**kw):
    """fcc 5x5x5 (500 sites, 125 cells: the two-word lattice path), three species."""
    cfg = cases.fcc32("double", composition={"Ti": 167, "Al": 167, "Nb": 166}, **kw)
    cfg["structure"]["supercell"] = [5, 5, 5]
    return cfg


def _senary(**kw):
    """fcc 3x3x3 (108 sites) with six species: the eight-species lattice kernel."""
    return cases.quinary("double", composition={e: 18 for e in ("Ti", "Al", "Nb", "V", "Zr", "Hf")}, **kw)


def mix():
    """Uneven jobs: sizes, species, shells, modes, precisions and kernels differ."""
    return [
        _fcc555(iterations=30000, seed=8, keep=3),
        _senary(iterations=30000, seed=9, keep=4),
        cases.fcc32("double", iterations=300000, seed=1, pair_weights=None),
        cases.quinary("double", iterations=40000, seed=2),
        cases.settings_16("single"),
        cases.rocksalt_split("double", iterations=60000, seed=4),
        cases.fcc32("single", composition={"Ti": 5, "Al": 27}, iteration_mode="systematic", seed=None,
                    iterations=None, keep=3, pair_weights=None),
        cases.quinary("single", cells=(2, 2, 3), iterations=70000, seed=6, keep=4),
        cases.fcc32("double", iterations=5000, seed=7, keep=2),
    ]


def records(run, c, d):
    L = N.lib()
    n = int(L.sqsg_run_count(run))
    T = np.float64 if int(c.prec) == 1 else np.float32
    nsp = sum(len(x.species_packed) for x in d)
    nsro = sum(x.prefactors.size for x in d)
    obj = np.zeros(max(n, 1), T)
    sp = np.zeros(max(n, 1) * nsp, np.uint8)
    sro = np.zeros(max(n, 1) * nsro, T)
    ids = np.zeros(max(n, 1), np.uint64)
    N.check(L.sqsg_run_copy(run, 0, n, N.ptr(obj), None, N.ptr(sp), N.ptr(sro), N.ptr(ids)))
    return (obj[:n].tobytes(), sp[: n * nsp].tobytes(), sro[: n * nsro].tobytes(), ids[:n].tobytes(),
            tuple(cases.run_levels(run)))


def alone(cfgs):
    out = []
    for cfg in cfgs:
        c = S.parse_config(cfg)
        d = S.prepare(c)
        job, keep = build_job(c, d)
        run = C.c_void_p()
        N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
        out.append(records(run, c, d))
        N.lib().sqsg_run_free(run)
    return out


def test_batch_equals_alone():
    cfgs = mix()
    ref = alone(cfgs)
    prepared = [(S.parse_config(cfg),) for cfg in cfgs]
    prepared = [(c, S.prepare(c)) for (c,) in prepared]
    jobs = (N.SqsgJob * len(cfgs))()
    keep = []
    for k, (c, d) in enumerate(prepared):
        job, bufs = build_job(c, d)
        jobs[k] = job
        keep.append(bufs)
    runs = (C.c_void_p * len(cfgs))()
    N.check(N.lib().sqsg_optimize_batch(jobs, len(cfgs), C.cast(runs, C.POINTER(C.c_void_p))))
    for k, (c, d) in enumerate(prepared):
        assert records(runs[k], c, d) == ref[k], k
        N.lib().sqsg_run_free(runs[k])


def test_served_equals_alone_with_overlapping_arrivals():
    cfgs = mix() * 2
    ref = alone(cfgs)
    with S.Server(0) as srv:
        prepared = [(c, S.prepare(c)) for c in (S.parse_config(cfg) for cfg in cfgs)]
        tickets = [None] * len(cfgs)

        def submitter():
            for k, (c, d) in enumerate(prepared):
                tickets[k] = srv.submit(None, prepared=(c, d))
                time.sleep(0.002 * (k % 3))  # arrivals while earlier jobs run

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for k, (c, d) in enumerate(prepared):
            run = srv.wait_run(tickets[k], timeout=120)
            assert records(run, c, d) == ref[k], k
            st = N.SqsgStatistics()
            N.check(N.lib().sqsg_run_statistics(run, C.byref(st)))
            assert st.timings_ns[0] > 0  # latency recorded
            N.lib().sqsg_run_free(run)
        stats = srv.stats()
        assert stats["completed"] == len(cfgs) and stats["pending"] == 0 and stats["active"] == 0


def test_served_admission_waits_for_memory():
    """A tiny arena holds one job at a time: later jobs wait for memory, then complete correctly."""
    cfgs = [cases.fcc32("double", iterations=200000, seed=s, pair_weights=None) for s in range(4)]
    ref = alone(cfgs)
    c0 = S.parse_config(cfgs[0])
    with S.Server(0, arena_bytes=12 << 20, default_max_results=65536) as srv:
        tickets = [srv.submit(cfg) for cfg in cfgs]
        for k, t in enumerate(tickets):
            run = srv.wait_run(t, timeout=120)
            c = S.parse_config(cfgs[k])
            assert records(run, c, S.prepare(c)) == ref[k]
            N.lib().sqsg_run_free(run)
    del c0


def test_served_rerun_after_overflow():
    """Jobs whose best levels hold more configurations than their candidate buffer (256) run again with the
    exact threshold, requeued as soon as they are collected; the results equal sqsg_optimize's alone."""
    cfgs = [cases.fcc32("double", iterations=200000, seed=s, pair_weights=None) for s in (11, 12, 13)]
    ref = alone(cfgs)
    with S.Server(0, default_max_results=256) as srv:
        tickets = [srv.submit(cfg) for cfg in cfgs]
        for k, t in enumerate(tickets):
            run = srv.wait_run(t, timeout=120)
            c = S.parse_config(cfgs[k])
            assert records(run, c, S.prepare(c)) == ref[k]
            N.lib().sqsg_run_free(run)
        st = srv.stats()
    assert st["completed"] == 3 and st["admitted"] > 3  # every job overflowed once


def test_server_rejects_jobs_that_never_fit():
    with S.Server(0, arena_bytes=1 << 20) as srv:
        with pytest.raises(N.NativeError) as e:
            srv.submit(cases.fcc32("double", iterations=1000, seed=1, max_results_per_objective=None))
        assert e.value.status_name == "SQSG_ERR_CAPACITY"


def test_served_result_pack_api():
    with S.Server(0) as srv:
        t = srv.submit(cases.settings_16("double"))
        pack = srv.result(t, timeout=60)
    assert pack.num_results() == 12870


def test_served_mixed_stream_equals_plain():
    """A short mixed stream (all six cells, 2-5 species, 2-4 shells, systematic and random jobs) served with
    overlapping arrivals returns, job by job, exactly what sqsg_optimize returns for the job alone."""
    import bench

    stream = bench.mixed_jobs(40, seed=7, rate=2000.0, budget=(1e5, 1e6))
    prepared = [(arr, S.parse_config(cfg)) for arr, cfg in stream]
    prepared = [(arr, c, S.prepare(c)) for arr, c in prepared]
    ref = []
    for _, c, d in prepared:
        job, keep = build_job(c, d)
        run = C.c_void_p()
        N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
        ref.append(records(run, c, d))
        N.lib().sqsg_run_free(run)
    with S.Server(0) as srv:
        t0 = time.perf_counter()
        tickets = []
        for arr, c, d in prepared:
            lag = arr - (time.perf_counter() - t0)
            if lag > 0:
                time.sleep(lag)
            tickets.append(srv.submit(None, prepared=(c, d)))
        for k, (_, c, d) in enumerate(prepared):
            run = srv.wait_run(tickets[k], timeout=300)
            assert records(run, c, d) == ref[k], k
            N.lib().sqsg_run_free(run)
        assert srv.stats()["launches"] >= 1


def test_server_kernels_leave_when_idle():
    """The ring's CTAs give up after a bounded number of empty polls (claim_live's idle limit): once
    the last job is done, no persistent launch of the server stays on the GPU."""
    import time as _time

    with S.Server(0) as srv:
        pack = srv.result(srv.submit(cases.fcc32("double", iterations=300000, seed=5)), timeout=120)
        assert pack.num_results() > 0
        running = C.c_uint32(1)
        deadline = _time.monotonic() + 5.0
        while _time.monotonic() < deadline:
            N.check(N.lib().sqsg_server_running(srv._h, C.byref(running)))
            if running.value == 0:
                break
            _time.sleep(0.005)
        assert running.value == 0
        # a job submitted after the kernels left starts a new launch and completes
        pack = srv.result(srv.submit(cases.settings_16("double")), timeout=120)
        assert pack.num_results() == 12870
