"""GPU parity: every configuration the device evaluates against the oracle, result sets against the
oracle's restated result collection, and the reference's own behavioural tests on the GPU path."""
import collections
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

import cases
import oracle
import sqsgenerator_b200 as S
from sqsgenerator_b200 import _native as N
from sqsgenerator_b200.optimize import build_job

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def require_device():
    assert N.device_count() > 0, "GPU tests need a CUDA device; the optimiser has no CPU path"


def native_run(config, **job_overrides):
    """Run a configuration through sqsg_optimize; returns (config, data, records dict, levels, info)."""
    c = S.parse_config(config)
    assert not isinstance(c, S.ParseError), c
    d = S.prepare(c)
    job, bufs = build_job(c, d)
    for k, v in job_overrides.items():
        setattr(job, k, v)
    run = C.c_void_p()
    N.check(N.lib().sqsg_optimize(C.byref(job), C.byref(run)))
    try:
        L = N.lib()
        n = int(L.sqsg_run_count(run))
        T = np.float64 if int(c.prec) == 1 else np.float32
        nsp = sum(len(x.species_packed) for x in d)
        nsro = sum(x.prefactors.size for x in d)
        obj = np.zeros(max(n, 1), T)
        sub = np.zeros(max(n, 1) * len(d), T)
        sp = np.zeros(max(n, 1) * nsp, np.uint8)
        sro = np.zeros(max(n, 1) * nsro, T)
        ids = np.zeros(max(n, 1), np.uint64)
        N.check(L.sqsg_run_copy(run, 0, n, N.ptr(obj), N.ptr(sub), N.ptr(sp), N.ptr(sro), N.ptr(ids)))
        st = N.SqsgStatistics()
        N.check(L.sqsg_run_statistics(run, C.byref(st)))
        cand = C.c_uint64()
        trunc = C.c_int32()
        exact = C.c_int32()
        N.check(L.sqsg_run_info(run, C.byref(cand), C.byref(trunc), C.byref(exact)))
        recs = dict(objective=obj[:n], sub=sub[: n * len(d)].reshape(n, len(d)), species=sp[: n * nsp].reshape(n, nsp),
                    sro=sro[: n * nsro].reshape(n, nsro), id=ids[:n], finished=int(st.finished))
        return c, d, recs, cases.run_levels(run), dict(candidates=cand.value, truncated=bool(trunc.value),
                                                         levels_exact=bool(exact.value))
    finally:
        N.lib().sqsg_run_free(run)


# --------------------------------------------------------------------------- per-configuration parity
@pytest.mark.parametrize("prec", ["double", "single"])
def test_trace_systematic_16_every_rank(prec):
    cfg = cases.settings_16(prec)
    c, d, pack, sp, bd, ob, ids = cases.trace(cfg, 13000)
    assert len(ob) == 12870
    assert sorted(ids.tolist()) == list(range(1, 12871))
    assert cases.trace_mismatches(d, sp, bd, ob, prec) == []
    for k in range(0, 12870, 97):  # rank -> configuration equals the reference's unrank
        exp = oracle.unrank_permutation(d[0].species_packed, int(ids[k]))
        assert np.array_equal(sp[k], exp)


@pytest.mark.parametrize("prec", ["double", "single"])
def test_trace_random_fcc32(prec):
    c, d, pack, sp, bd, ob, ids = cases.trace(cases.fcc32(prec, iterations=20000), 20000)
    assert len(ob) == 20000
    assert cases.trace_mismatches(d, sp, bd, ob, prec) == []
    # every evaluated configuration is a permutation of the packed species (Fisher-Yates)
    assert np.all(np.sort(sp, axis=1) == np.sort(d[0].species_packed))


@pytest.mark.parametrize("prec", ["double", "single"])
def test_trace_quinary_k5(prec):
    c, d, pack, sp, bd, ob, ids = cases.trace(cases.quinary(prec, iterations=4000), 4000)
    assert cases.trace_mismatches(d, sp, bd, ob, prec) == []


@pytest.mark.parametrize("prec", ["double", "single"])
def test_trace_split_two_sublattices(prec):
    c, d, pack, sp, bd, ob, ids = cases.trace(cases.rocksalt_split(prec, iterations=4000), 4000)
    assert len(d) == 2
    assert cases.trace_mismatches(d, sp, bd, ob, prec) == []


def test_trace_interact_two_windows():
    """Interact mode with two sublattices: each window is shuffled inside itself (shuffle.h:41-49)."""
    cfg = cases.rocksalt_split("double", iterations=3000)
    cfg["sublattice_mode"] = "interact"
    cfg["shell_weights"] = {"1": 1.0, "2": 0.5}
    cfg["seed"] = 11
    c, d, pack, sp, bd, ob, ids = cases.trace(cfg, 3000)
    assert len(d[0].windows) == 2
    assert cases.trace_mismatches(d, sp, bd, ob, "double") == []
    for lo, hi in d[0].windows:
        assert np.all(np.sort(sp[:, lo:hi], axis=1) == np.sort(d[0].species_packed[lo:hi]))


# --------------------------------------------------------------------------- reference tests on the GPU
@pytest.mark.parametrize("prec", ["single", "double"])
def test_systematic_all_results(prec):
    """python/tests/test_core.py:45-67"""
    config = S.parse_config(cases.settings_16(prec))
    results = S.optimize(config)
    assert config.iterations == 12870
    assert results.num_results() == config.iterations
    ranks = set(range(1, config.iterations + 1))
    site_coords = {i: tuple(np.round(c, 5)) for i, c, _ in config.structure()}
    for _, rset in results:
        for sol in rset:
            st = sol.structure()
            assert math.isclose(sol.objective, 0.0)
            assert collections.Counter(st.species) == collections.Counter({22: 8, 13: 8})
            ranks.discard(int(sol.rank()))
            for i, c, _ in st:
                assert tuple(np.round(c, 5)) == site_coords[i]
    assert not ranks


@pytest.mark.parametrize("prec", ["single", "double"])
def test_systematic_all_results_partial(prec):
    """python/tests/test_core.py:82-128 — only the H sites of a 32-site cell are permuted."""
    s = cases.settings_16(prec)
    s["structure"] = dict(lattice=np.diag([1, 2, 3]).tolist(),
                          coords=[[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5]],
                          species=[1, 2] * 2, supercell=[2, 2, 2])
    config = S.parse_config(s)
    results = S.optimize(config)
    assert results.num_results() == config.iterations == 12870
    cs = config.structure()
    random_sites = {i for i, _, z in cs if z == 1}
    assert len(random_sites) == 16
    for _, rset in results:
        for sol in rset:
            st = sol.structure()
            assert math.isclose(sol.objective, 0.0)
            assert collections.Counter(st.species) == collections.Counter({22: 8, 13: 8, 2: 16})
            assert {i for i, z in enumerate(st.species) if z in (22, 13)} == random_sites


def _check_bonds_one_minus_sro(results, config):
    """python/tests/test_core.py:209-249 — recount bonds from an independent pair list."""
    first = results.best()
    st = first.structure()
    sm = st.shell_matrix(config.shell_radii[0], 1.0e-3)
    w = config.shell_weights[0]
    pairs = [(i, j, int(sm[i, j])) for i in range(len(st)) for j in range(i) if int(sm[i, j]) in w]
    shell_map = {s: i for i, s in enumerate(w)}
    species_map = {v: i for i, v in enumerate(sorted(set(st.species)))}
    hist = collections.Counter(s for *_, s in pairs)
    K = len(species_map)
    for _, sols in results:
        sol = sols[0]
        sros = np.zeros((len(shell_map), K, K))
        species = sol.species
        for i, j, s in pairs:
            sros[shell_map[s], species_map[species[i]], species_map[species[j]]] += 1
        for i in range(K):
            for j in range(i + 1, K):
                tot = sros[:, i, j] + sros[:, j, i]
                sros[:, i, j] = tot
                sros[:, j, i] = tot
        for k, (bonds, sro) in enumerate(zip(sros, sol.sro())):
            nb = sum(bonds[a, b] for a in range(K) for b in range(a, K))
            assert hist[{v: s for s, v in shell_map.items()}[k]] == nb
            assert np.allclose(bonds, 1 - sro)


@pytest.mark.parametrize("prec", ["single", "double"])
@pytest.mark.parametrize("mode", ["systematic", "random"])
def test_bonds_correct_one_sublattice(prec, mode):
    """python/tests/test_core.py:252-271"""
    s = cases.settings_16(prec)
    del s["pair_weights"]
    s.update(prefactors=1, iteration_mode=mode, iterations=15000)
    config = S.parse_config(s)
    _check_bonds_one_minus_sro(S.optimize(config), config)


@pytest.mark.parametrize("prec", ["single", "double"])
def test_bonds_correct_one_sublattice_non_exhaustive(prec):
    """python/tests/test_core.py:274-288"""
    s = cases.settings_16(prec)
    del s["pair_weights"]
    s.update(prefactors=1, iteration_mode="random", iterations=1200)
    s["structure"]["species"] = [1, 1, 2, 2]
    s["structure"]["supercell"] = [2, 2, 2]
    s["composition"] = {"sites": "He", "Ti": 6, "Al": 5, "O": 5}
    config = S.parse_config(s)
    _check_bonds_one_minus_sro(S.optimize(config), config)


@pytest.mark.parametrize("prec", ["single", "double"])
def test_random_seed_reproducible(prec):
    """python/tests/test_core.py:291-317"""
    s = cases.settings_16(prec)
    s.update(iteration_mode="random", iterations=500, seed=42)
    a, b = S.optimize(S.parse_config(s)), S.optimize(S.parse_config(s))
    assert a.config.seed == b.config.seed == [42]
    key = lambda p: collections.Counter((round(float(x.objective), 12), tuple(x.structure().species))  # noqa: E731
                                        for _, rs in p for x in rs)
    assert key(a) == key(b)


# --------------------------------------------------------------------------- result sets vs the oracle
def _oracle_core(d, res, keep):
    """The reference's deterministic result core: every configuration at or below the (keep+1)-th
    best distinct objective of the restated collection."""
    objs = sorted({float(r["objective"]) for r in res})
    tstar = objs[keep] if len(objs) > keep else math.inf
    return {(r["species"][0].tobytes(), r["objective"].tobytes(), r["sro"][0].tobytes())
            for r in res if float(r["objective"]) <= tstar}


@pytest.mark.parametrize("prec", ["double", "single"])
@pytest.mark.parametrize("keep", [1, 3, 10, 64, 100])
def test_systematic_result_set_equals_oracle(prec, keep):
    """fcc 2x2x2 A4B28 (35,960 permutations) with default pair weights: the device result set equals
    the restated reference collection's deterministic core, bit for bit (species, objective, sro)."""
    cfg = cases.fcc32(prec, composition={"Ti": 4, "Al": 28}, iteration_mode="systematic", keep=keep,
                      seed=None, iterations=None, pair_weights=None)
    c, d, recs, levels, info = native_run(cfg)
    assert recs["finished"] == 35960 and not info["truncated"] and info["levels_exact"]
    res, _ = oracle.optimize(d, prec=prec, iteration_mode="systematic", iterations=35960, keep=keep)
    T = np.float64 if prec == "double" else np.float32
    gpu = {(recs["species"][k].tobytes(), T(recs["objective"][k]).tobytes(), recs["sro"][k].astype(T).tobytes())
           for k in range(len(recs["objective"]))}
    assert len(gpu) == len(recs["objective"])
    assert gpu == _oracle_core(d, res, keep)
    lv = oracle.systematic_levels(d[0], prec=prec, keep=keep)
    assert levels == lv


def test_random_records_bit_exact_and_deduplicated():
    c, d, recs, levels, info = native_run(cases.fcc32("double", iterations=200000, pair_weights=None))
    n = len(recs["objective"])
    assert n > 0 and not info["truncated"]
    keys = {recs["species"][k].tobytes() for k in range(n)}
    assert len(keys) == n
    for k in range(0, n, max(1, n // 300)):
        o, sro = oracle.evaluate(d[0], recs["species"][k], "double")
        assert o.tobytes() == recs["objective"][k].tobytes()
        assert sro.tobytes() == recs["sro"][k].reshape(sro.shape).tobytes()
    # the result set holds exactly the keep+1 best distinct objectives
    distinct = sorted(set(recs["objective"].tolist()))
    assert distinct == [v for v, _, _ in levels][: len(distinct)]
    assert len(distinct) == 11


@pytest.mark.parametrize("cell,prec,keep,cap", [("fcc32", "double", 3, None), ("fcc32", "double", 10, 7),
                                                ("fcc32", "single", 5, 2), ("fcc32", "double", 64, None),
                                                ("fcc32", "single", 100, 3), ("quinary", "double", 100, None),
                                                ("quinary", "single", 64, 1), ("quinary", "double", 1023, None)])
def test_random_result_set_from_full_trace(cell, prec, keep, cap):
    """Every evaluation of a random run is traced; the result set must equal the rule restated here on
    the trace: the keep+1 smallest distinct objectives, one record per distinct configuration (the
    smallest id), ordered by objective then id, at most cap+1 per objective. keep >= 32 exercises the
    warps' best lists in shared memory (the reference accepts any keep, io/config/combined.h:164-174)."""
    if cell == "fcc32":
        n = 120000
        cfg = cases.fcc32(prec, iterations=n, seed=11, keep=keep)
    else:
        n = 30000
        cfg = cases.quinary(prec, iterations=n, seed=12, keep=keep)
    if cap is not None:
        cfg["max_results_per_objective"] = cap
    _, d, _, sp, _, ob, ids = cases.trace(cfg, n)
    assert len(ob) == n
    levels = sorted(set(ob.tolist()))[: keep + 1]
    lset = set(levels)
    order = sorted((float(ob[k]), int(ids[k]), k) for k in range(len(ob)) if float(ob[k]) in lset)
    seen, per, expect = set(), collections.Counter(), []
    for o, i, k in order:
        key = sp[k].tobytes()
        if key in seen:
            continue
        seen.add(key)
        if cap is not None and per[o] > cap:
            continue
        per[o] += 1
        expect.append((o, i, key))
    _, _, recs, lv, info = native_run(cfg)
    got = [(float(recs["objective"][k]), int(recs["id"][k]), recs["species"][k].tobytes())
           for k in range(len(recs["objective"]))]
    assert not info["truncated"] and info["levels_exact"]
    assert [v for v, _, _ in lv] == levels
    assert got == expect


def test_split_records_bit_exact():
    c, d, recs, levels, info = native_run(cases.rocksalt_split("double", iterations=50000, seed=9))
    n = len(recs["objective"])
    assert n > 0
    for k in range(n):
        tot = None
        off = 0
        for p, part in enumerate(d):
            sp = recs["species"][k, off:off + len(part.species_packed)]
            off += len(part.species_packed)
            o, _ = oracle.evaluate(part, sp, "double")
            assert o == recs["sub"][k, p]
            tot = o if tot is None else tot + o
        assert tot.tobytes() == recs["objective"][k].tobytes()


def test_max_results_per_objective():
    """All 12,870 configurations of the 16-site cell have objective 0: with a cap of 5 the result set
    is the 6 configurations of smallest rank (the reference's `>` test admits cap + 1)."""
    cfg = cases.settings_16("double")
    cfg["max_results_per_objective"] = 5
    c, d, recs, levels, info = native_run(cfg)
    assert recs["objective"].tolist() == [0.0] * 6
    assert recs["id"].tolist() == [1, 2, 3, 4, 5, 6]
    for k in range(6):
        assert np.array_equal(recs["species"][k], oracle.unrank_permutation(d[0].species_packed, k + 1))


def test_cancel_via_callback():
    seen = []

    def cb(ctx):
        seen.append(ctx.statistics.finished)
        ctx.stop()

    cfg = cases.fcc32("double", iterations=2_000_000_000, chunk_size=1_000_000, pair_weights=None)
    pack = S.optimize(cfg, callback=cb)
    assert seen and pack.statistics.finished < 2_000_000_000
    assert pack.num_results() > 0


def test_unsupported_sizes_are_errors():
    cfg = cases.fcc32("double", iterations=1000, keep=2000)
    with pytest.raises(N.NativeError) as e:
        S.optimize(cfg)
    assert e.value.status_name == "SQSG_ERR_UNSUPPORTED"


# --------------------------------------------------------------------------- full size
@pytest.mark.slow
@pytest.mark.parametrize("prec", ["double", "single"])
def test_fcc32_systematic_full_space_levels(prec):
    """All 601,080,390 permutations of the fcc 2x2x2 A16B16 cell: the keep+1 best objectives, the
    exact number of configurations at each and an order-independent checksum of their ranks equal
    the oracle's exhaustive enumeration (tests/golden/fcc32_systematic_levels.json)."""
    golden = json.load(open(os.path.join(GOLDEN, "fcc32_systematic_levels.json")))
    cfg = cases.fcc32(prec, iteration_mode="systematic", seed=None, iterations=None)
    c, d, recs, levels, info = native_run(cfg)
    assert recs["finished"] == golden["num_permutations"]
    exp = [(g["objective"], g["count"], g["checksum"]) for g in golden[prec]]
    assert levels == exp
    assert info["levels_exact"]
    # the returned records are optimal or near-optimal configurations, each bit-exact
    for k in range(0, len(recs["objective"]), max(1, len(recs["objective"]) // 200)):
        o, _ = oracle.evaluate(d[0], recs["species"][k], prec)
        assert o.tobytes() == recs["objective"][k].tobytes()
        assert oracle.rank_permutation(recs["species"][k]) == int(recs["id"][k])


# --------------------------------------------------------------------------- RNG stream and fast path
@pytest.mark.parametrize("composition,floyd", [({"Ti": 16, "Al": 16}, 1), ({"Ti": 16, "Al": 16}, 0),
                                               ({"Ti": 7, "Al": 25}, 1), ({"Ti": 11, "Al": 11, "Nb": 10}, 1)],
                         ids=["binary_fast_path_floyd", "binary_fast_path_fisher_yates", "binary_skewed_floyd",
                              "ternary_general_path"])
def test_random_stream_is_philox_fisher_yates(composition, floyd):
    """Configuration g is the shuffle of the packed initial arrangement with xoshiro128** words seeded by
    the Philox block of counter g (tests/philox_ref.py) — Fisher-Yates, or Floyd's sampling of the rarer
    species on a two-species window: it depends on (seed, g) alone, not on tiles, launches or devices."""
    import philox_ref

    total = 2_097_153
    cfg = cases.fcc32("double", composition=composition, iterations=total, seed=0x1234_5678_9ABC)
    with N.options(binary_floyd=floyd):
        c, d, pack, sp, bd, ob, ids = cases.trace(cfg, total)
    assert np.array_equal(ids, np.arange(total, dtype=np.uint64))
    windows = [tuple(w) for w in d[0].windows.tolist()]
    rng = np.random.default_rng(0)
    for g in sorted(set(rng.choice(total, size=400, replace=False).tolist()) | {0, 1, total - 1}):
        conf = d[0].species_packed.tolist()
        philox_ref.shuffle(conf, windows, cfg["seed"], g, 0, floyd=bool(floyd))
        assert conf == sp[g].tolist(), g
    assert cases.trace_mismatches(d, sp[:1500], bd[:1500], ob[:1500], "double") == []


def test_random_results_do_not_depend_on_the_split():
    """Three contiguous shares of a seeded random job (as on three GPUs) evaluate exactly the
    configurations of the whole job: merged levels equal the whole job's levels."""
    from sqsgenerator_b200.shard import merge_levels, shard_range

    cfg = cases.fcc32("double", iterations=3_000_001, seed=77, pair_weights=None)
    _, _, _, whole, _ = native_run(cfg)
    parts = []
    for r in range(3):
        first, count = shard_range(3_000_001, 3, r)
        _, _, _, lv, _ = native_run(cfg, range_first=first, range_count=count)
        parts.append(lv)
    assert merge_levels(parts, 10) == whole


def test_fast_path_64_sites():
    cfg = cases.fcc32("double", iterations=20000, pair_weights=None)
    cfg["structure"]["supercell"] = [2, 2, 4]
    cfg["composition"] = {"Ti": 32, "Al": 32}
    c, d, pack, sp, bd, ob, ids = cases.trace(cfg, 20000)
    assert len(d[0].species_packed) == 64
    assert cases.trace_mismatches(d, sp, bd, ob, "double") == []


@pytest.mark.parametrize("prec", ["double", "single"])
def test_fast_path_sites_of_different_degree(prec):
    """Perovskite positions, one binary composition over all 40 sites: shell 1 has sites of degree 0, 2
    and 6, shell 2 of degree 0 and 12, so the bit-mask path's degree classes (all but the largest,
    with wrapped negative coefficients) carry the mixed-pair count."""
    cfg = dict(prec=prec, structure=dict(lattice=(np.eye(3) * 4.0).tolist(),
                                         coords=[[0, 0, 0], [0.5, 0.5, 0.5], [0.5, 0.5, 0], [0.5, 0, 0.5],
                                                 [0, 0.5, 0.5]],
                                         species=[1] * 5, supercell=[2, 2, 2]),
               composition={"Ti": 20, "Al": 20}, shell_weights={"1": 1.0, "2": 0.5}, iterations=4000, seed=11,
               thread_config=1, keep=10)
    c, d, pack, sp, bd, ob, ids = cases.trace(cfg, 4000)
    assert len(d[0].species_packed) == 40 and len(ob) == 4000
    assert cases.trace_mismatches(d, sp, bd, ob, prec) == []


@pytest.mark.parametrize("prec", ["double", "single"])
def test_fast_path_partial_window_systematic(prec):
    """A 20-site window inside a 64-site cell of the same background species (two species overall)."""
    cfg = cases.fcc32(prec, iteration_mode="systematic", seed=None, iterations=None, keep=4, pair_weights=None)
    cfg["structure"]["supercell"] = [2, 2, 4]
    cfg["structure"]["species"] = [1] * 4
    cfg["composition"] = {"sites": list(range(20)), "Ti": 10, "H": 10}
    c, d, pack, sp, bd, ob, ids = cases.trace(cfg, 184756)
    assert c.iterations == 184756 and len(ob) == 184756
    assert sorted(ids.tolist()) == list(range(1, 184757))
    rows = np.random.default_rng(1).choice(184756, size=3000, replace=False)
    assert cases.trace_mismatches(d, sp[rows], bd[rows], ob[rows], prec) == []
    for k in rows[:200]:
        exp = oracle.unrank_permutation(d[0].species_packed[d[0].windows[0][0]:d[0].windows[0][1]], int(ids[k]))
        lo, hi = d[0].windows[0]
        got = sp[k, lo:hi]
        uniq = sorted(set(d[0].species_packed[lo:hi].tolist()))
        assert np.array_equal(got, np.array([uniq[x] for x in exp], np.uint8))
    c2, d2, recs, levels, info = native_run(cfg)
    lv = oracle.systematic_levels(d2[0], prec=prec, keep=4)
    assert levels == lv
