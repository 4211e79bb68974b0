"""The allocation-free entry point against the regular one.

sqsg_optimize_levels_noalloc serves callers that cannot allocate device memory (a host framework that
owns the device budget through its own pool, a process whose memory is capped once work starts): it
keeps its scratch in a static device array instead of calling cudaMalloc. Two calls in a row must
report exactly the objective levels (values, counts, id checksums) and statistics that sqsg_optimize
reports for the same job — the arithmetic is integer counting plus the same floating-point objective,
so the tolerance is zero. This file is collected last so that a failure here stops a run only after
every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import cases
import sqsgenerator_b200 as S
from sqsgenerator_b200 import _native as N
from sqsgenerator_b200.optimize import build_job

pytestmark = pytest.mark.gpu


def regular(job):
    run = C.c_void_p()
    N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
    try:
        st = N.SqsgStatistics()
        N.check(N.lib().sqsg_run_statistics(run, C.byref(st)))
        return cases.run_levels(run), int(st.finished)
    finally:
        N.lib().sqsg_run_free(run)


def noalloc(job):
    cap = 1100
    n = C.c_uint32(cap)
    v = np.zeros(cap, np.float64)
    cnt = np.zeros(cap, np.uint64)
    cs = np.zeros(cap, np.uint64)
    st = N.SqsgStatistics()
    err = C.create_string_buffer(256)
    status = N.lib().sqsg_optimize_levels_noalloc(C.byref(job), None, C.byref(n), N.ptr(v), N.ptr(cnt), N.ptr(cs),
                                                  C.byref(st), err, len(err))
    return status, err.value.decode(), [(float(v[i]), int(cnt[i]), int(cs[i])) for i in range(n.value)], int(st.finished)


CASES = {
    "systematic_16_double": lambda: cases.settings_16("double"),
    "systematic_fcc32_a4b28_single": lambda: cases.fcc32("single", composition={"Ti": 4, "Al": 28},
                                                         iteration_mode="systematic", seed=None, iterations=None,
                                                         keep=5),
    "random_fcc32_double": lambda: cases.fcc32("double", iterations=300000, seed=17),
    "random_split_double": lambda: cases.rocksalt_split("double", iterations=50000, seed=5),
    "random_quinary_keep100_double": lambda: cases.quinary("double", iterations=40000, seed=8, keep=100),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_noalloc_matches_regular_entry_twice(name):
    assert N.device_count() > 0, "needs a CUDA device"
    c = S.parse_config(CASES[name]())
    d = S.prepare(c)
    job, keep_alive = build_job(c, d)
    ref_levels, ref_finished = regular(job)
    assert ref_levels
    for _ in range(2):  # the static scratch keeps the previous call's contents
        status, msg, levels, finished = noalloc(job)
        assert status == 0, msg
        assert finished == ref_finished
        assert levels == ref_levels


def test_noalloc_rejects_jobs_beyond_its_limits():
    assert N.device_count() > 0, "needs a CUDA device"
    c = S.parse_config(cases.fcc32("double", iterations=10 ** 18, seed=3))
    d = S.prepare(c)
    job, keep_alive = build_job(c, d)
    status, msg, levels, finished = noalloc(job)
    assert N.STATUS_NAMES[status] == "SQSG_ERR_CAPACITY"
    assert "tile" in msg
