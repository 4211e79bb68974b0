"""GPU parity at the sizes the benchmark configurations name, on every evaluation path.

Every configuration the device evaluates in these runs is traced and checked against the oracle:
ordered bond counts (core/optimization.h:74-77) bit for bit and the objective (optimization.h:79-103)
bit for bit in the run's precision. Each test also asserts which path the library chose
(sqsg_plan_job), so that the general pair-stream path in each of its forms (narrow stream staged in
shared memory, narrow stream read through L1, wide stream for cells above 512 sites), the bit-mask
path and the lattice path are each covered, and the paths are checked against each other.
"""
import collections
import ctypes as C

import numpy as np
import pytest

import cases
import oracle
import sqsgenerator_b200 as S
from sqsgenerator_b200 import _native as N
from sqsgenerator_b200.optimize import build_job

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def require_device():
    assert N.device_count() > 0, "GPU tests need a CUDA device; the optimiser has no CPU path"


def plan_of(cfg):
    c = S.parse_config(cfg)
    assert not isinstance(c, S.ParseError), c
    d = S.prepare(c)
    job, bufs = build_job(c, d)
    return N.plan(job)


def traced(cfg, n, prec):
    c, d, pack, sp, bd, ob, ids = cases.trace(cfg, n)
    assert len(ob) == n
    bad = cases.trace_mismatches(d, sp, bd, ob, prec)
    assert bad == [], bad[:5]
    return c, d, sp, ob, ids


def fcc(cells, composition, shells, prec="double", iterations=2000, seed=5, **kw):
    weights = {str(k): 1.0 / k for k in range(1, shells + 1)}
    cfg = dict(prec=prec, structure=dict(lattice=(np.eye(3) * 4.0).tolist(), coords=cases.fcc_coords(),
                                         species=[1] * 4, supercell=list(cells)),
               composition=composition, shell_weights=weights, iterations=iterations, seed=seed,
               thread_config=1, keep=5)
    cfg.update(kw)
    return cfg


def config3(prec="double", iterations=3000):
    """fcc 4x4x4 (256 sites), A52B51C51D51E51, 3 shells (12/6/24 neighbours, P = 5376), weights 1/0.5/0.25."""
    return cases.quinary(prec, cells=(4, 4, 4), iterations=iterations, seed=0, keep=10,
                         composition={"Ti": 52, "Al": 51, "Nb": 51, "V": 51, "Zr": 51})


def config4(prec="double", iterations=3000):
    """rocksalt 3x3x3 (216 sites) split: Ti54Al54 cations and N96B12 anions, 2 shells per sublattice."""
    return cases.rocksalt_split(prec, cells=(3, 3, 3), iterations=iterations, seed=1,
                                composition=[{"sites": "Na", "Ti": 54, "Al": 54}, {"sites": "Cl", "N": 96, "B": 12}])


PATHS = {"lattice": {"use_tuning": 0}, "general": {"force_general": 1}}  # the rules' path, not the table's


@pytest.mark.parametrize("path", sorted(PATHS))
@pytest.mark.parametrize("prec", ["double", "single"])
def test_config3_quinary_256_sites(prec, path):
    """In trace mode the lattice path also runs the pair stream: the traced bonds are the pair
    stream's, and any configuration whose lattice objective differs is an error of the call."""
    cfg = config3(prec)
    with N.options(**PATHS[path]):
        p = plan_of(cfg)
        assert p["parts"][0]["path"] == path
        if path == "general":
            assert p["parts"][0]["stream_narrow"] and p["parts"][0]["stream_staged"]
        c, d, sp, ob, ids = traced(cfg, 3000, prec)
    assert len(d[0].species_packed) == 256 and len(d[0].pairs) == 5376
    assert collections.Counter(sp[0].tolist()) == collections.Counter(d[0].species_packed.tolist())


@pytest.mark.parametrize("path", sorted(PATHS))
@pytest.mark.parametrize("prec", ["double", "single"])
def test_config4_rocksalt_split_216_sites(prec, path):
    cfg = config4(prec)
    with N.options(**PATHS[path]):
        p = plan_of(cfg)
        assert [x["path"] for x in p["parts"]] == [path, path]
        assert not p["parts"][0]["stream_staged"] and not p["parts"][1]["stream_staged"]
        c, d, sp, ob, ids = traced(cfg, 3000, prec)
    assert [len(x.species_packed) for x in d] == [108, 108]
    assert [len(x.pairs) for x in d] == [972, 972]


LATTICE_CASES = {
    "config3": lambda: config3("double", iterations=200000),
    "config4": lambda: config4("single", iterations=300000),
    "fcc32_ternary": lambda: cases.fcc32("double", composition={"Ti": 11, "Al": 11, "Nb": 10}, iterations=300000,
                                         seed=4),
    "fcc32_systematic_ternary": lambda: cases.fcc32("double", composition={"Ti": 2, "Al": 3, "Nb": 27},
                                                    iteration_mode="systematic", seed=None, iterations=None, keep=6,
                                                    pair_weights=None),
    "perovskite_333": lambda: dict(prec="double", structure=dict(
        lattice=(np.eye(3) * 4.0).tolist(), coords=[[0, 0, 0], [0.5, 0.5, 0.5], [0.5, 0.5, 0], [0.5, 0, 0.5],
                                                    [0, 0.5, 0.5]], species=[1] * 5, supercell=[3, 3, 3]),
        composition={"Ti": 45, "Al": 45, "Nb": 45}, shell_weights={"1": 1.0, "2": 0.5}, iterations=100000, seed=11,
        thread_config=1, keep=7),
    "rocksalt_interact": lambda: dict(cases.rocksalt_split("double", cells=(3, 3, 3), iterations=100000, seed=2,
                                                           composition=[{"sites": "Na", "Ti": 54, "Al": 54},
                                                                        {"sites": "Cl", "N": 96, "B": 12}]),
                                      sublattice_mode="interact", shell_weights={"1": 1.0, "2": 0.5}),
    "bcc_4x4x2_quaternary": lambda: dict(prec="single", structure=dict(
        lattice=(np.eye(3) * 2.87).tolist(), coords=[[0, 0, 0], [0.5, 0.5, 0.5]], species=[1] * 2,
        supercell=[4, 4, 2]), composition={"Ti": 16, "Al": 16, "Nb": 16, "V": 16},
        shell_weights={"1": 1.0, "2": 0.5, "3": 0.25}, iterations=200000, seed=21, thread_config=1, keep=9),
    # 65-128 cells: two-word cell sets (sqsg_engine_latw)
    "fcc500_ternary_4shells": lambda: fcc((5, 5, 5), {"Ti": 167, "Al": 167, "Nb": 166}, 4, iterations=60000, seed=41,
                                          keep=6),
    "bcc250_quinary": lambda: dict(prec="double", structure=dict(
        lattice=(np.eye(3) * 2.87).tolist(), coords=[[0, 0, 0], [0.5, 0.5, 0.5]], species=[1] * 2,
        supercell=[5, 5, 5]), composition={"Ti": 50, "Al": 50, "Nb": 50, "V": 50, "Zr": 50},
        shell_weights={"1": 1.0, "2": 0.5, "3": 0.25}, iterations=60000, seed=42, thread_config=1, keep=5),
    "fcc_445_quaternary_single": lambda: fcc((4, 4, 5), {"Ti": 80, "Al": 80, "Nb": 80, "V": 80}, 3, prec="single",
                                             iterations=60000, seed=43, keep=4),
    "fcc500_binary": lambda: fcc((5, 5, 5), {"Ti": 250, "Al": 250}, 2, iterations=60000, seed=44, keep=5),
    "rocksalt_445_split": lambda: cases.rocksalt_split("double", cells=(4, 4, 5), iterations=40000, seed=45, keep=4,
                                                      composition=[{"sites": "Na", "Ti": 160, "Al": 160},
                                                                   {"sites": "Cl", "N": 280, "B": 40}]),
    # six and eight species: the eight-species variant of the lattice path (sqsg_engine_lat)
    "fcc_333_senary": lambda: fcc((3, 3, 3), {"Ti": 18, "Al": 18, "Nb": 18, "V": 18, "Zr": 18, "Hf": 18}, 2,
                                  iterations=100000, seed=31, keep=5),
    "bcc_444_octonary": lambda: dict(prec="double", structure=dict(
        lattice=(np.eye(3) * 2.87).tolist(), coords=[[0, 0, 0], [0.5, 0.5, 0.5]], species=[1] * 2,
        supercell=[4, 4, 4]), composition={e: 16 for e in ("Ti", "Al", "Nb", "V", "Zr", "Hf", "Ta", "Mo")},
        shell_weights={"1": 1.0, "2": 0.5}, iterations=100000, seed=32, thread_config=1, keep=4),
}

# the lattice kernel of each case: binary parts, at most five species, at most eight
LATTICE_KERNELS = {"config3": "sqsg_engine_lat5", "config4": "sqsg_engine_lat2", "fcc32_ternary": "sqsg_engine_lat5",
                   "fcc32_systematic_ternary": "sqsg_engine_lat5", "perovskite_333": "sqsg_engine_lat5",
                   "rocksalt_interact": "sqsg_engine_lat5", "bcc_4x4x2_quaternary": "sqsg_engine_lat5",
                   "fcc_333_senary": "sqsg_engine_lat", "bcc_444_octonary": "sqsg_engine_lat",
                   "fcc500_ternary_4shells": "sqsg_engine_latw", "bcc250_quinary": "sqsg_engine_latw",
                   "fcc_445_quaternary_single": "sqsg_engine_latw", "fcc500_binary": "sqsg_engine_latw",
                   "rocksalt_445_split": "sqsg_engine_latw"}


@pytest.mark.parametrize("name", sorted(LATTICE_CASES))
def test_lattice_and_general_paths_agree(name):
    """The same job on the lattice path and on the pair-stream path: the same result set (objectives,
    ids, species, SRO) and the same exact objective levels."""
    cfg = LATTICE_CASES[name]()
    with N.options(use_tuning=0):  # the rules' path (the tuning table may prefer the pair stream)
        plan = plan_of(cfg)
        assert [x["path"] for x in plan["parts"]] == ["lattice"] * len(plan["parts"])
        assert plan["kernel"] == LATTICE_KERNELS[name]
        a = _full_records(cfg)
    with N.options(force_general=1):
        assert plan_of(cfg)["parts"][0]["path"] == "general"
        b = _full_records(cfg)
    assert a[0] > 0 and a == b


@pytest.mark.parametrize("name", ["fcc32_ternary", "perovskite_333", "bcc_4x4x2_quaternary", "rocksalt_interact",
                                  "fcc_333_senary", "bcc_444_octonary", "fcc500_ternary_4shells", "bcc250_quinary",
                                  "fcc_445_quaternary_single"])
def test_lattice_trace_against_oracle(name):
    cfg = dict(LATTICE_CASES[name]())
    cfg["iterations"] = 4000
    with N.options(use_tuning=0):
        assert plan_of(cfg)["parts"][0]["path"] == "lattice"
        traced(cfg, 4000, cfg["prec"])


def test_narrow_stream_read_through_l1_fcc500():
    """fcc 5x5x5 (500 sites), three species, four shells (12/6/24/12 neighbours): staging the stream
    would cost a CTA per SM, so it is read from the job blob through L1."""
    cfg = fcc((5, 5, 5), {"Ti": 167, "Al": 167, "Nb": 166}, 4, iterations=1500)
    with N.options(force_general=1):  # the cell would take the two-word lattice path
        p = plan_of(cfg)
        assert p["parts"][0]["path"] == "general"
        assert p["parts"][0]["stream_narrow"] and not p["parts"][0]["stream_staged"]
        c, d, sp, ob, ids = traced(cfg, 1500, "double")
    assert len(d[0].species_packed) == 500


def test_wide_stream_above_512_sites_fcc864():
    """fcc 6x6x6 (864 sites): column offsets above 16 bits take the wide stream form."""
    cfg = fcc((6, 6, 6), {"Ti": 432, "Al": 432}, 2, iterations=1000)
    p = plan_of(cfg)  # 216 cells: general path
    assert p["parts"][0]["path"] == "general" and not p["parts"][0]["stream_narrow"]
    c, d, sp, ob, ids = traced(cfg, 1000, "double")
    assert len(d[0].species_packed) == 864


@pytest.mark.parametrize("prec", ["double", "single"])
def test_bitmask_and_general_paths_agree_fcc32(prec):
    """The same random job on the bit-mask path and, forced, on the general path: the same
    configurations, the same objectives and the same result set."""
    cfg = cases.fcc32(prec, iterations=50000, seed=19, pair_weights=None)
    assert plan_of(cfg)["parts"][0]["path"] == "bitmask"
    _, _, sp_a, ob_a, ids_a = traced(cfg, 50000, prec)
    with N.options(force_general=1):
        assert plan_of(cfg)["parts"][0]["path"] == "general"
        _, _, sp_b, ob_b, ids_b = traced(cfg, 50000, prec)
    order_a, order_b = np.argsort(ids_a), np.argsort(ids_b)
    assert np.array_equal(ids_a[order_a], ids_b[order_b])
    assert np.array_equal(sp_a[order_a], sp_b[order_b])
    assert ob_a[order_a].tobytes() == ob_b[order_b].tobytes()


def _full_records(cfg):
    c = S.parse_config(cfg)
    d = S.prepare(c)
    job, bufs = build_job(c, d)
    run = C.c_void_p()
    N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
    try:
        n = int(N.lib().sqsg_run_count(run))
        T = np.float64 if int(c.prec) == 1 else np.float32
        nsp = sum(len(x.species_packed) for x in d)
        nsro = sum(x.prefactors.size for x in d)
        obj = np.zeros(max(n, 1), T)
        sp = np.zeros(max(n, 1) * nsp, np.uint8)
        sro = np.zeros(max(n, 1) * nsro, T)
        ids = np.zeros(max(n, 1), np.uint64)
        N.check(N.lib().sqsg_run_copy(run, 0, n, N.ptr(obj), None, N.ptr(sp), N.ptr(sro), N.ptr(ids)))
        return (n, obj[:n].tobytes(), sp[: n * nsp].tobytes(), sro[: n * nsro].tobytes(), ids[:n].tobytes(),
                tuple(cases.run_levels(run)))
    finally:
        N.lib().sqsg_run_free(run)


def _records(cfg):
    c = S.parse_config(cfg)
    d = S.prepare(c)
    job, bufs = build_job(c, d)
    run = C.c_void_p()
    N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
    try:
        n = int(N.lib().sqsg_run_count(run))
        T = np.float64 if int(c.prec) == 1 else np.float32
        obj = np.zeros(max(n, 1), T)
        ids = np.zeros(max(n, 1), np.uint64)
        N.check(N.lib().sqsg_run_copy(run, 0, n, N.ptr(obj), None, None, None, N.ptr(ids)))
        return [(float(obj[k]), int(ids[k])) for k in range(n)], cases.run_levels(run)
    finally:
        N.lib().sqsg_run_free(run)


@pytest.mark.parametrize("keep,cap", [(3, 2), (5, 1), (2, 7)])
def test_max_results_per_objective_follows_the_rule(keep, cap):
    """Systematic fcc 2x2x2 A4B28 (35,960 ranks): the result set is, for each of the keep+1 best
    distinct objectives, the cap+1 configurations of smallest rank (the reference's `>` test admits
    one more than max_results_per_objective, sqs.h:423-426), ordered by objective then rank."""
    cfg = cases.fcc32("double", composition={"Ti": 4, "Al": 28}, iteration_mode="systematic", keep=keep,
                      seed=None, iterations=None, pair_weights=None, max_results_per_objective=cap)
    _, d, _, sp, _, ob, ids = cases.trace(cfg, 35960)
    assert len(ob) == 35960
    levels = sorted(set(ob.tolist()))[: keep + 1]
    expect = []
    for v in levels:
        rows = sorted(int(ids[k]) for k in np.flatnonzero(ob == v))
        expect += [(v, r) for r in rows[: cap + 1]]
    got, lv = _records(cfg)
    assert [x for x, _, _ in lv] == levels
    assert got == expect


def test_staging_wait_runs_out_and_the_context_stays_usable():
    """The device's bounded wait for a job's staged data: with the debug option that issues no copy,
    every CTA gives up after the bound, the call returns SQSG_ERR_TIMEOUT, and the next call on the
    same context runs normally. No fault and no hang: the wait is bounded by the global timer."""
    cfg = cases.fcc32("double", iterations=100000, seed=3)
    with N.options(debug_skip_staging=1, stage_wait_ns=20_000_000):
        with pytest.raises(N.NativeError) as e:
            _records(cfg)
        assert e.value.status_name == "SQSG_ERR_TIMEOUT"
    with N.options(debug_skip_staging=1, stage_wait_ns=20_000_000, force_general=1):
        with pytest.raises(N.NativeError) as e:
            _records(cfg)
        assert e.value.status_name == "SQSG_ERR_TIMEOUT"
    got, lv = _records(cfg)
    assert got and lv


def test_plan_reports_occupancy_on_the_device():
    p = plan_of(config3())
    assert p["kernel"] == "sqsg_engine_lat5" and p["ctas_per_sm"] >= 1
    with N.options(force_general=1):
        p = plan_of(config3())
    assert p["kernel"] == "sqsg_engine_wide" and p["ctas_per_sm"] >= 1
    p = plan_of(cases.fcc32("double"))
    assert p["kernel"] == "sqsg_engine_mask" and p["ctas_per_sm"] >= 1


def test_autotune_records_a_choice_and_results_do_not_change():
    """sqsg_autotune measures the launch choices of a job's bucket and records the fastest; a job of
    that bucket then follows it (sqsg_plan_job says so), with the same result set as under the rules."""
    cfg = LATTICE_CASES["fcc32_ternary"]()
    c = S.parse_config(cfg)
    d = S.prepare(c)
    job, bufs = build_job(c, d)
    with N.options(use_tuning=0):
        ref = _full_records(cfg)
        assert not N.plan(job)["tuned"]
    best, tried = N.autotune(job, 0.5)
    assert tried and best["configs_per_s"] == max(t["configs_per_s"] for t in tried)
    assert {t["path"] for t in tried} == {"lattice", "general"}
    assert N.plan(job)["tuned"]
    assert _full_records(cfg) == ref
