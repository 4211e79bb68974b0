#!/usr/bin/env python
"""Benchmark of the B200 SQS optimisation hot path (one JSON line on stdout, rank 0).

Workload (default ``systematic``): exhaustive enumeration of the fcc 2x2x2 (32-site, a = 4.0 A)
A16B16 cell, all C(32,16) = 601,080,390 permutations by rank, shells 1/2 weighted 1.0/0.5, all pair
weights 1, target 0, keep 10, float64 objective. One step = one ``sqsg_optimize`` call over the whole
rank space (split into contiguous rank ranges across ranks when N > 1).

``value``: configurations per second of the engine kernel (CUDA events around the launch, inputs
resident); ``e2e``: the same through the C ABI with host buffers (job upload, launch, result download
and selection inside the timed region). ``--impl reference`` times the restated reference CPU loop
(the oracle) on the host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import threading
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "configs/sec on 1 B200 (served/batched vs plain GPU); p50/p99 SQS job latency"
SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def workload_config(name: str):
    import cases

    if name == "systematic":
        return cases.fcc32("double", iteration_mode="systematic", seed=None, iterations=None), (
            "fcc 2x2x2 (32 sites) A16B16 systematic, all 601,080,390 permutations, 2 shells (12/3 neighbours, "
            "P=240 pairs), weights 1.0/0.5, pair weights 1, keep 10, float64")
    if name == "random":
        return cases.fcc32("double", iterations=1_000_000, seed=42), (
            "fcc 2x2x2 (32 sites) A16B16 random, 1e6 random configurations (Floyd sampling of the 16 B sites, Philox-seeded xoshiro128** words), 2 shells, weights 1.0/0.5, "
            "pair weights 1, keep 10, float64")
    if name == "quinary":
        return cases.quinary("double", cells=(4, 4, 4), iterations=20_000_000, seed=0, keep=10,
                             composition={"Ti": 52, "Al": 51, "Nb": 51, "V": 51, "Zr": 51}), (
            "fcc 4x4x4 (256 sites) A52B51C51D51E51 random, 3 shells (12/6/24, P=5376), weights 1.0/0.5/0.25, "
            "64 independent chains of 2e7 configurations (seeds 0..63) in one batched launch, float64")
    if name == "split":
        return cases.rocksalt_split("double", cells=(3, 3, 3), iterations=500_000_000, seed=1,
                                    composition=[{"sites": "Na", "Ti": 54, "Al": 54}, {"sites": "Cl", "N": 96, "B": 12}]), (
            "rocksalt 3x3x3 (216 sites) split: Ti54Al54 cations and N96B12 anions optimised together, 2 shells per "
            "sublattice (P=648+324 each), weights 1.0/0.5, 5e8 configurations (Floyd sampling: 54 + 12 draws "
            "each), float64")
    if name == "split_single":
        return cases.rocksalt_split("single", cells=(3, 3, 3), iterations=500_000_000, seed=1,
                                    composition=[{"sites": "Na", "Ti": 54, "Al": 54}, {"sites": "Cl", "N": 96, "B": 12}]), (
            "rocksalt 3x3x3 (216 sites) split: Ti54Al54 cations and N96B12 anions optimised together, 2 shells per "
            "sublattice (P=648+324 each), weights 1.0/0.5, 5e8 configurations (Floyd sampling: 54 + 12 draws "
            "each), float32")
    if name == "fcc500":
        cfg = cases.fcc32("double", composition={"Ti": 167, "Al": 167, "Nb": 166}, iterations=20_000_000, seed=5,
                          shell_weights={"1": 1.0, "2": 0.5, "3": 1.0 / 3, "4": 0.25}, keep=10)
        cfg["structure"]["supercell"] = [5, 5, 5]
        return cfg, ("fcc 5x5x5 (500 sites) A167B167C166 random, 4 shells (12/6/24/12, P=13500), weights 1/k, "
                     "2e7 configurations, float64 (the largest cell of the served mixed stream)")
    raise SystemExit(f"unknown workload {name}")


# Served mixed-job stream: (lattice kind, repetitions) -> fcc 32/108/256/500 and bcc 54/128 sites.
MIXED_CELLS = (("fcc", 2), ("bcc", 3), ("fcc", 3), ("bcc", 4), ("fcc", 4), ("fcc", 5))
MIXED_ELEMENTS = ("Ti", "Al", "Nb", "V", "Zr")


def _cell(kind: str, rep: int):
    if kind == "fcc":
        a, coords = 4.0, [[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]
    else:
        a, coords = 2.87, [[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]]
    return dict(lattice=(np.eye(3) * a).tolist(), coords=coords, species=[1] * len(coords), supercell=[rep] * 3), \
        len(coords) * rep ** 3


def mixed_jobs(n: int, seed: int = 2026, rate: float = 200.0, budget=(1e5, 1e8)):
    """The mixed-job stream: Poisson arrivals (rate jobs/s); cells drawn uniformly from fcc 32, bcc 54, fcc 108,
    bcc 128, fcc 256 and fcc 500 sites; 2-5 species with positive integer counts summing to the site count; 2-4
    shells with weights 1/k; random budgets log-uniform in ``budget``; 10 % systematic fcc 32-site binary jobs
    (minority 3-7 atoms). Returns [(arrival seconds, reference-schema config dict)]."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        shells = int(rng.integers(2, 5))
        weights = {str(k): 1.0 / k for k in range(1, shells + 1)}
        if rng.random() < 0.1:
            structure, _ = _cell("fcc", 2)
            m = int(rng.integers(3, 8))
            cfg = dict(prec="double", iteration_mode="systematic", structure=structure,
                       composition={"Ti": m, "Al": 32 - m}, shell_weights=weights, keep=10)
        else:
            kind, rep = MIXED_CELLS[int(rng.integers(len(MIXED_CELLS)))]
            structure, n_sites = _cell(kind, rep)
            k = int(rng.integers(2, 6))
            cuts = np.sort(rng.choice(np.arange(1, n_sites), k - 1, replace=False))
            counts = np.diff(np.concatenate([[0], cuts, [n_sites]])).astype(int)
            iters = int(10 ** rng.uniform(np.log10(budget[0]), np.log10(budget[1])))
            cfg = dict(prec="double", iteration_mode="random", structure=structure,
                       composition={e: int(c) for e, c in zip(MIXED_ELEMENTS, counts)}, shell_weights=weights,
                       iterations=iters, seed=int(rng.integers(1 << 62)), thread_config=1, keep=10)
        out.append((t, cfg))
    return out


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML read every 5 ms from a
    thread, with one sample taken on entry and one on exit so that even a region of a few
    milliseconds has two; nvidia-smi at 200 ms when NVML is not importable. Read-only."""

    # NVML clocks-event reason bits (nvml.h): sw power cap, hw slowdown, sw thermal, hw thermal
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int):
        self.device = device
        self.rows = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.util = []  # NVML utilization.gpu samples (percent of time a kernel ran)
        self.nvml = None
        self.proc = None
        self.path = None
        self._stop = threading.Event()
        self._thread = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:  # noqa: BLE001 — fall back to the NVML index
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _sample(self):
        nv, h = self.nvml
        try:
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                              float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)), int(get_reasons(h))))
            self.util.append(float(nv.nvmlDeviceGetUtilizationRates(h).gpu))
        except Exception:  # noqa: BLE001 — a failed read is a missing sample
            pass

    def _loop(self):
        while not self._stop.wait(0.005):
            self._sample()

    def __enter__(self):
        try:
            self.nvml = self._handle()
        except Exception:  # noqa: BLE001
            self.nvml = None
        if self.nvml:
            self._sample()
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()
            return self
        try:
            self.path = tempfile.mktemp(suffix=".csv")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={SMI_FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.nvml:
            self._sample()
            self._stop.set()
            self._thread.join(timeout=5)
            return
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for line in open(self.path):
                r = [p.strip() for p in line.split(",")]
                if len(r) >= 9 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                    bits = sum(self.REASON_BITS[names[k]] for k in range(4) if r[5 + k].lower() == "active")
                    self.rows.append((float(r[1]), float(r[2]), bits))

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [r[0] for r in self.rows]
        mx = max(r[1] for r in self.rows)
        reasons = sorted({n for r in self.rows for n, b in self.REASON_BITS.items() if r[2] & b})
        loaded = [v for v in sm if v > 0.5 * mx] or sm
        out = {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "samples": len(self.rows),
               "source": "nvml" if self.nvml else "nvidia-smi", "reasons": reasons}
        if self.util:
            out["util_mean"] = statistics.mean(self.util)
        return out


def cpu_sample(seconds: float, keep: int, workload: str = "systematic"):
    """The restated reference loop (oracle, on oracle geometry for the systematic cell) over a bounded
    sample, all host threads. Returns (configurations, seconds, threads, description)."""
    import cases
    import oracle

    threads = os.cpu_count() or 1
    if workload == "systematic":
        sd = cases.oracle_fcc32()
        t = time.perf_counter()
        oracle.systematic_levels(sd, keep=keep, threads=threads, first=0, count=2_000_000)
        rate = 2_000_000 / (time.perf_counter() - t)
        count = int(min(rate * seconds, 601_080_390))
        t = time.perf_counter()
        oracle.systematic_levels(sd, keep=keep, threads=threads, first=0, count=count)
        dt = time.perf_counter() - t
        return count, dt, threads, (
            f"ranks 1..{count} (contiguous prefix) of the 601,080,390-rank space through the restated reference loop "
            f"(unrank + count_bonds + compute_objective + next_permutation) on {threads} threads; the result "
            "collection is replaced by per-objective counting")
    import sqsgenerator_b200 as S

    cfg, _ = workload_config(workload)
    c = S.parse_config(cfg)
    d = S.prepare(c)
    mode = "split" if workload.startswith("split") else "interact"
    prec = "double" if int(c.prec) == 1 else "single"
    probe = 20_000
    t = time.perf_counter()
    oracle.optimize(d, prec=prec, iterations=probe, keep=c.keep, threads=threads, sublattice_mode=mode)
    rate = probe / (time.perf_counter() - t)
    count = max(probe, int(rate * seconds))
    t = time.perf_counter()
    _, st = oracle.optimize(d, prec=prec, iterations=count, keep=c.keep, threads=threads, sublattice_mode=mode)
    dt = time.perf_counter() - t
    return count, dt, threads, (
        f"{count} random configurations through the restated reference optimizer loop (rapidrand shuffler shared by "
        f"{threads} threads, chunk 100000, result collection) of the same structure")


def run_reference(args):
    """--impl reference: the oracle's restatement of the reference CPU path on this host's cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg, desc = workload_config(args.workload)
    per_step = []
    for step in range(args.warmup + args.steps):
        count, dt, threads, sample = cpu_sample(args.ref_seconds, cfg["keep"], args.workload)
        if step >= args.warmup:
            per_step.append((count, dt))
    configs = sum(x[0] for x in per_step)
    secs = sum(x[1] for x in per_step)
    value = configs / secs
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "configs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / len(per_step) * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc},
            "cpu_baseline": {"value": value, "unit": "configs/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "configs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def check_records(d, prec: str, recs) -> dict:
    """Checker of the cpu_baseline leg: the objective of each sampled record recomputed by the oracle
    (restated reference count_bonds + compute_objective, parts summed left to right) must equal the
    device's bit for bit."""
    import oracle

    T = np.float64 if prec == "double" else np.float32
    ok = 0
    for species, obj in recs:
        tot, off = None, 0
        for part in d:
            n = len(part.species_packed)
            o, _ = oracle.evaluate(part, species[off:off + n], prec)
            off += n
            tot = o if tot is None else T(tot + o)
        ok += int(np.asarray(tot, T).tobytes() == np.asarray(obj, T).tobytes())
    return {"records_checked": len(recs), "records_bit_exact": ok}


def measure(workload: str, steps: int, warmup: int, device: int, world: int, rank: int, max_results: int,
            limit: int = 0) -> dict:
    """One workload through sqsg_optimize (sqsg_optimize_batch for the 64 chains of the quinary
    workload): `warmup` untimed steps, then `steps` timed steps with an L2 flush before each."""
    import torch

    import cases as _cases
    import sqsgenerator_b200 as S
    from sqsgenerator_b200 import _native as N
    from sqsgenerator_b200.optimize import build_job
    from sqsgenerator_b200.shard import shard_range

    cfg, desc = workload_config(workload)
    c = S.parse_config(cfg)
    d = S.prepare(c)
    n_jobs = 64 if workload.startswith("quinary") else 1
    per_job = c.iterations if not limit else min(limit, c.iterations)
    first, count = shard_range(per_job, world, rank)
    jobs = (N.SqsgJob * n_jobs)()
    keep_alive = []
    for k in range(n_jobs):
        ck = S.parse_config(dict(cfg, seed=k)) if n_jobs > 1 else c
        job, bufs = build_job(ck, d, device=device)
        job.range_first, job.range_count, job.max_results = first, count, max_results
        jobs[k] = job
        keep_alive.append(bufs)
    L = N.lib()
    P_total = sum(len(x.pairs) for x in d)
    nsp = sum(len(x.species_packed) for x in d)
    nsro = sum(x.prefactors.size for x in d)
    T = np.float64 if int(c.prec) == 1 else np.float32
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")

    def step():
        runs = (C.c_void_p * n_jobs)()
        t0 = time.perf_counter()
        if n_jobs == 1:
            N.check(L.sqsg_optimize(C.byref(jobs[0]), C.cast(runs, C.POINTER(C.c_void_p))))
        else:
            N.check(L.sqsg_optimize_batch(jobs, n_jobs, C.cast(runs, C.POINTER(C.c_void_p))))
        results, sample = 0, []
        t_copy = time.perf_counter()
        for k in range(n_jobs):
            run = runs[k]
            n = int(L.sqsg_run_count(run))
            obj = np.empty(max(n, 1), T)
            sp = np.empty(max(n, 1) * nsp, np.uint8)
            sro = np.empty(max(n, 1) * nsro, T)
            ids = np.empty(max(n, 1), np.uint64)
            N.check(L.sqsg_run_copy(run, 0, n, N.ptr(obj), None, N.ptr(sp), N.ptr(sro), N.ptr(ids)))
            results += n
            if k == 0:
                rows = sp[: n * nsp].reshape(n, nsp)
                pick = np.unique(np.linspace(0, max(n - 1, 0), num=min(n, 64)).astype(np.int64)) if n else []
                sample = [(rows[i].copy(), obj[i]) for i in pick]
        wall = time.perf_counter() - t0
        copy_s = time.perf_counter() - t_copy
        finished = h2d = d2h = 0
        for k in range(n_jobs):
            st = N.SqsgStatistics()
            N.check(L.sqsg_run_statistics(runs[k], C.byref(st)))
            finished += int(st.finished)
            a, b = C.c_uint64(), C.c_uint64()
            N.check(L.sqsg_run_transfer(runs[k], C.byref(a), C.byref(b)))
            h2d += a.value
            d2h += b.value
            if k == 0:
                loop = st.timings_ns[2] * 1e-9
        stages = N.run_stages(runs[0])
        stages["copy_to_caller"] = copy_s
        levels = _cases.run_levels(runs[0])
        info_c, info_t, info_e = C.c_uint64(), C.c_int32(), C.c_int32()
        N.check(L.sqsg_run_info(runs[0], C.byref(info_c), C.byref(info_t), C.byref(info_e)))
        for k in range(n_jobs):
            L.sqsg_run_free(runs[k])
        return dict(wall=wall, loop=loop, finished=finished, results=results, h2d=h2d, d2h=d2h, levels=levels,
                    sample=sample, stages=stages, truncated=bool(info_t.value))

    for _ in range(warmup):
        step()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    out = []
    with ClockSampler(device) as clk:
        for _ in range(steps):
            flush.fill_(1)  # L2 flush between timed steps (256 MiB > 126 MB L2)
            torch.cuda.synchronize()
            out.append(step())
        torch.cuda.synchronize()
    plan = N.plan(jobs[0])
    return dict(workload=workload, desc=desc, config=c, data=d, n_jobs=n_jobs, total=per_job * n_jobs,
                P_total=P_total, nsp=nsp, steps=steps, out=out, clocks=clk.summary(), plan=plan,
                loop=sum(o["loop"] for o in out), wall=sum(o["wall"] for o in out),
                finished=sum(o["finished"] for o in out))


def roofline_of(res: dict, smem_bw: float, int_rate: float, world: int = 1, popc_rate: float | None = None) -> dict:
    """Roofline of the dominant kernel, per launch (CUDA-event time) against the peaks measured in this run.

    Pair-stream and bit-mask paths: fixed algorithmic work of 2*P shared-memory species bytes (P pairs)
    and 3*P integer operations per configuration. Lattice path: it reads no species per pair; its work
    is one 64-bit AND-popcount per (translation class, species pair a <= b < K-1), i.e. two 32-bit
    population counts per unit (plan: lattice_units), against the measured popcount rate. The 2*P
    figure is kept beside it (smem_equiv_frac) to compare the paths on one scale."""
    launch_s = res["loop"] / res["steps"]
    configs_per_launch = res["finished"] / res["steps"] / world
    P = res["P_total"]
    achieved = 2 * P * configs_per_launch / launch_s / 1e9
    prof = os.path.join(ROOT, "profiles", f"sqsg_engine_{res['workload']}.json")
    traffic, traffic_case = None, None
    if os.path.exists(prof):
        pj = json.load(open(prof))
        traffic, traffic_case = pj.get("dram_bytes_per_launch"), pj.get("case")
    common = {"traffic": traffic, "traffic_case": traffic_case,
              "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum of one launch (ncu), scaled to this "
                              "launch's configurations where the capture ran a smaller case (traffic_case)",
              "int32_frac": (3 * P * configs_per_launch / launch_s) / int_rate, "int32_peak_ops": int_rate,
              "kernel": res["plan"]["kernel"], "paths": [p["path"] for p in res["plan"]["parts"]],
              "ctas_per_sm": res["plan"]["ctas_per_sm"]}
    parts = res["plan"]["parts"]
    if popc_rate and parts and all(p["path"] == "lattice" for p in parts):
        units = sum(p["lattice_units"] for p in parts)
        rate = 2 * units * configs_per_launch / launch_s  # 32-bit popcounts per second
        return dict({"bound": "popc", "achieved": rate / 1e9, "peak": popc_rate / 1e9, "unit": "Gpopc/s",
                     "frac": rate / popc_rate,
                     "peak_source": "measured in this run: independent AND-POPC-ADD chains (sqsg_microbench kind 2)",
                     "algorithmic": f"2 x {units} 32-bit popcounts per configuration ({units} 64-bit AND-popcount "
                                    "units: translation classes x species pairs)",
                     "smem_equiv_frac": achieved / (smem_bw / 1e9)}, **common)
    return dict({"bound": "smem", "achieved": achieved, "peak": smem_bw / 1e9, "unit": "GB/s",
                 "frac": achieved / (smem_bw / 1e9),
                 "peak_source": "measured in this run: conflict-free LDS.32 microbenchmark (sqsg_microbench kind 0)",
                 "algorithmic": f"2*P = {2 * P} B of shared-memory species reads per configuration (P = {P} pairs)"},
                **common)


def extra_line(res: dict, smem_bw: float, int_rate: float, cpu: dict | None, parity: dict | None,
               popc_rate: float | None = None) -> dict:
    last = res["out"][-1]
    return {"workload": res["desc"], "value": res["finished"] / res["loop"], "unit": "configs/s",
            "steps": res["steps"], "ms_per_step": res["loop"] / res["steps"] * 1e3,
            "configs_per_step": res["finished"] // res["steps"],
            "e2e": {"value": res["finished"] / res["wall"], "unit": "configs/s", "h2d_bytes_per_step": last["h2d"],
                    "d2h_bytes_per_step": last["d2h"], "ms_per_step": res["wall"] / res["steps"] * 1e3,
                    "host_stages_s": last["stages"]},
            "roofline": roofline_of(res, smem_bw, int_rate, 1, popc_rate), "clocks": res["clocks"], "cpu_baseline": cpu,
            "parity": parity, "results": {"records_per_step": last["results"], "truncated": last["truncated"],
                                          "best_levels": last["levels"][:3]}}


def run_b200(args):
    import torch

    from sqsgenerator_b200 import _native as N
    from sqsgenerator_b200.shard import merge_levels

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    device = local
    torch.cuda.set_device(device)
    res = measure(args.workload, args.steps, args.warmup, device, world, rank, args.max_results, args.limit)
    loop, wall, finished = res["loop"], res["wall"], res["finished"]
    if world > 1:
        t = torch.tensor([loop, wall], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        loop, wall = t.tolist()
        f = torch.tensor([finished], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(f)
        finished = int(f.item())
        gathered = [None] * world
        torch.distributed.all_gather_object(gathered, res["out"][-1]["levels"])
    else:
        gathered = [res["out"][-1]["levels"]]
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    c = res["config"]
    levels = merge_levels(gathered, c.keep)  # exact: counts and checksum halves add up
    parity = None
    golden_path = os.path.join(ROOT, "tests", "golden", "fcc32_systematic_levels.json")
    if args.workload == "systematic" and not args.limit and os.path.exists(golden_path):
        g = json.load(open(golden_path))["double"]
        parity = {"levels_match_oracle": levels == [(x["objective"], x["count"], x["checksum"]) for x in g],
                  "best_objective": levels[0][0], "optimal_configurations": levels[0][1],
                  "source": "tests/golden/fcc32_systematic_levels.json (the oracle's exhaustive enumeration)"}
    smem_bw, _ = N.microbench(0, device)
    int_rate, _ = N.microbench(1, device)
    popc_rate, _ = N.microbench(2, device)
    res_w = dict(res, loop=loop, wall=wall, finished=finished)
    roofline = roofline_of(res_w, smem_bw, int_rate, world, popc_rate)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        n, dt, threads, sample = cpu_sample(args.cpu_seconds, c.keep, args.workload)
        cpu = {"value": n / dt, "unit": "configs/s", "cores": threads, "kind": "port", "sample": sample}
    last = res["out"][-1]
    line = {"metric": METRIC, "value": finished / loop, "unit": "configs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": loop / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": res["desc"], "configs_per_step": res["total"], "sites": res["nsp"],
                       "pairs": res["P_total"], "jobs": res["n_jobs"],
                       "l2": "flushed between timed steps (256 MiB device write)", "max_results": args.max_results,
                       "parallelism": f"configuration space split into {world} contiguous ranges"},
            "e2e": {"value": finished / wall, "unit": "configs/s", "h2d_bytes_per_step": last["h2d"],
                    "d2h_bytes_per_step": last["d2h"], "ms_per_step": wall / args.steps * 1e3,
                    "host_stages_s": last["stages"]},
            "roofline": roofline, "cpu_baseline": cpu, "clocks": res["clocks"], "gpu_launches": args.steps,
            "results": {"records_per_step": last["results"], "truncated": last["truncated"],
                        "truncation_note": "records are capped at max_results per step; the exact objective "
                                           "levels (counts and id checksums) cover the whole space",
                        "levels": levels[:3]},
            "parity": parity}
    if world == 1 and args.extras:
        extras = {}
        for name, steps in (("random", 20), ("quinary", 2), ("split", 2), ("split_single", 2), ("fcc500", 2)):
            r = measure(name, steps, 1, device, 1, 0, 0)
            cpu_x, par = None, None
            if not args.no_cpu_baseline:
                n, dt, threads, sample = cpu_sample(args.cpu_seconds / 2, r["config"].keep, name)
                cpu_x = {"value": n / dt, "unit": "configs/s", "cores": threads, "kind": "port", "sample": sample}
                prec = "double" if int(r["config"].prec) == 1 else "single"
                par = check_records(r["data"], prec, r["out"][-1]["sample"])
            extras[name] = extra_line(r, smem_bw, int_rate, cpu_x, par, popc_rate)
            line["gpu_launches"] += r["steps"] * (1 + 1)  # engine + rebuilt records per step
        import copy

        served_args = copy.copy(args)
        served_args.warmup = 1
        extras["served"] = served_measure(served_args, device, 1, 0, smem_bw)
        line["extras"] = extras
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def _run_digest(L, N, run, cases_mod):
    """Levels plus the selected records' objectives and ids of one run (for arm-to-arm parity)."""
    n = int(L.sqsg_run_count(run))
    st = N.SqsgStatistics()
    N.check(L.sqsg_run_statistics(run, C.byref(st)))
    ids = np.zeros(max(n, 1), np.uint64)
    obj = np.zeros(max(n, 1), np.float64)
    N.check(L.sqsg_run_copy(run, 0, n, N.ptr(obj), None, None, None, N.ptr(ids)))
    return dict(levels=tuple(cases_mod.run_levels(run)), ids=ids[:n].tobytes(), obj=obj[:n].tobytes(),
                finished=int(st.finished), latency_ns=int(st.timings_ns[0]))


def cpu_served_sample(prepared, seconds: float) -> dict:
    """cpu_baseline leg of the served stream: its jobs in arrival order through the restated reference
    loop (oracle) on all host cores, each cut to a bounded budget, until `seconds` have passed."""
    import oracle

    threads = os.cpu_count() or 1
    done = 0
    jobs = 0
    t0 = time.perf_counter()
    for _, c, d, _ in prepared:
        if time.perf_counter() - t0 > seconds:
            break
        if int(c.iteration_mode) == 1:
            n = min(int(c.iterations), 200_000)
            oracle.systematic_levels(d[0], keep=c.keep, threads=threads, first=0, count=n)
        else:
            n = min(int(c.iterations), 20_000)
            oracle.optimize(d, iterations=n, keep=c.keep, threads=threads, sublattice_mode="interact")
        done += n
        jobs += 1
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "configs/s", "cores": threads, "kind": "port",
            "sample": f"the first {jobs} jobs of the stream in arrival order, each cut to at most 20,000 random "
                      "configurations (200,000 ranks for systematic jobs), through the restated reference optimizer "
                      f"loop on {threads} threads"}


def served_measure(args, device: int, world: int, rank: int, smem_bw: float | None = None) -> dict | None:
    """The served mixed-job stream on one GPU: the same Poisson stream of jobs through (1) the plain path, one
    sqsg_optimize call at a time in arrival order (a FIFO queue in front of the GPU), (2) the continuous-batching
    server (sqsg_server_*), and (3) one offline sqsg_optimize_batch call over all jobs. Host precompute (parsing
    and geometry) is done before the timed region for every arm; job preparation, upload, kernels, result
    download and selection are inside it. Returns the result line (rank 0) or None."""
    import torch

    import cases as _cases
    import sqsgenerator_b200 as S
    from sqsgenerator_b200 import _native as N
    from sqsgenerator_b200.optimize import build_job

    L = N.lib()
    stream = mixed_jobs(args.jobs, seed=2026, rate=args.rate)[rank::world]  # each GPU serves its share
    prepared = []
    for arr, cfg in stream:
        c = S.parse_config(cfg)
        d = S.prepare(c)
        prepared.append((arr, c, d, sum(len(x.pairs) for x in d)))
    warm = [(0.0, c, d, P) for (_, c, d, P) in prepared[: min(8, len(prepared))]]

    # Every arm keeps its run handles (results already in host memory) and computes the parity digests
    # after its timed region: hashing multi-million-record result sets in Python is test work, and done
    # inline it held the interpreter while arrivals were due.
    def plain(items):
        t0 = time.perf_counter()
        lat, runs = [], []
        for arr, c, d, _ in items:
            now = time.perf_counter() - t0
            if now < arr:
                time.sleep(arr - now)
            job, bufs = build_job(c, d, device=device)
            run = C.c_void_p()
            N.check(L.sqsg_optimize(C.byref(job), C.byref(run)))
            lat.append(time.perf_counter() - t0 - arr)
            runs.append(run)
        span = time.perf_counter() - t0
        digests, kernel_s, host_s = [], 0.0, 0.0
        for run in runs:
            digests.append(_run_digest(L, N, run, _cases))
            st = N.run_stages(run)
            kernel_s += st["kernel"]
            host_s += st["total"] - st["wait"]
            L.sqsg_run_free(run)
        return span, lat, digests, kernel_s, host_s

    def served(items):
        srv = S.Server(device)
        try:
            n = len(items)
            tickets, sub_lag = [None] * n, [0.0] * n
            ready = [threading.Event() for _ in range(n)]
            t0 = time.perf_counter()

            def submitter():
                for k, (arr, c, d, _) in enumerate(items):
                    now = time.perf_counter() - t0
                    if now < arr:
                        time.sleep(arr - now)
                    tickets[k] = srv.submit(None, prepared=(c, d))
                    sub_lag[k] = time.perf_counter() - t0 - arr
                    ready[k].set()

            th = threading.Thread(target=submitter)
            th.start()
            runs = []
            for k in range(n):
                ready[k].wait()
                runs.append(srv.wait_run(tickets[k], timeout=600))
            th.join()
            span = time.perf_counter() - t0
            digests, lat = [], []
            for k, run in enumerate(runs):
                dg = _run_digest(L, N, run, _cases)
                digests.append(dg)
                lat.append(sub_lag[k] + dg["latency_ns"] * 1e-9)
                L.sqsg_run_free(run)
            return span, lat, digests, srv.stats()
        finally:
            srv.close()

    def batched(items):
        jobs = (N.SqsgJob * len(items))()
        keep = []
        for k, (_, c, d, _) in enumerate(items):
            job, bufs = build_job(c, d, device=device)
            jobs[k] = job
            keep.append(bufs)
        runs = (C.c_void_p * len(items))()
        t0 = time.perf_counter()
        N.check(L.sqsg_optimize_batch(jobs, len(items), C.cast(runs, C.POINTER(C.c_void_p))))
        span = time.perf_counter() - t0
        digests = [_run_digest(L, N, runs[k], _cases) for k in range(len(items))]
        for k in range(len(items)):
            L.sqsg_run_free(runs[k])
        return span, digests

    for _ in range(args.warmup):  # library, kernel attributes, workspaces and the server's rings warm up
        plain(warm)
        served(warm)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(device) as clk:
        with ClockSampler(device) as clk_p:
            p_span, p_lat, p_dig, p_kernel, p_host = plain(prepared)
        with ClockSampler(device) as clk_s:
            s_span, s_lat, s_dig, s_stats = served(prepared)
        with ClockSampler(device) as clk_b:
            b_span, b_dig = batched(prepared)
    configs = sum(x["finished"] for x in p_dig)
    pair_evals = sum(x["finished"] * P for x, (_, _, _, P) in zip(p_dig, prepared))
    same = sum(1 for a, b in zip(p_dig, s_dig) if (a["levels"], a["ids"], a["obj"]) == (b["levels"], b["ids"], b["obj"]))
    same_b = sum(1 for a, b in zip(p_dig, b_dig) if (a["levels"], a["ids"], a["obj"]) == (b["levels"], b["ids"], b["obj"]))
    spans = [p_span, s_span, b_span]
    if world > 1:
        t = torch.tensor(spans, dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        spans = t.tolist()
        f = torch.tensor([configs, pair_evals, same, same_b, len(prepared)], dtype=torch.float64,
                         device=f"cuda:{device}")
        torch.distributed.all_reduce(f)
        configs, pair_evals, same, same_b, n_jobs = (int(v) for v in f.tolist())
        lat_all = [None] * world
        torch.distributed.all_gather_object(lat_all, (p_lat, s_lat))
        p_lat = [v for a, _ in lat_all for v in a]
        s_lat = [v for _, b in lat_all for v in b]
    else:
        n_jobs = len(prepared)
    p_span, s_span, b_span = spans
    if rank != 0:
        return None
    if smem_bw is None:
        smem_bw, _ = N.microbench(0, device)
    cpu = None if args.no_cpu_baseline or world > 1 else cpu_served_sample(prepared, args.cpu_seconds)
    q = lambda v, p: float(np.percentile(np.asarray(v), p)) * 1e3  # noqa: E731
    value = configs / s_span
    achieved = 2 * pair_evals / s_span / 1e9
    return {"metric": METRIC, "value": value, "unit": "configs/s", "n_gpus": world, "steps": 1,
            "warmup": args.warmup, "ms_per_step": s_span * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"served mixed-job stream: {n_jobs} jobs, Poisson arrivals at {args.rate}/s "
                                   "(seed 2026); cells fcc32/bcc54/fcc108/bcc128/fcc256/fcc500, 2-5 species, 2-4 "
                                   "shells weights 1/k, random budgets log-uniform 1e5-1e8, 10% systematic fcc32",
                       "jobs": n_jobs, "configs": configs, "pair_evaluations": pair_evals,
                       "l2": "not flushed: every job's data is uploaded from host memory inside the timed region"},
            "served": {"configs_per_s": value, "makespan_s": s_span, "p50_ms": q(s_lat, 50), "p99_ms": q(s_lat, 99),
                       "launches": s_stats["launches"], "gpu_util_mean": clk_s.summary().get("util_mean")},
            "plain": {"configs_per_s": configs / p_span, "makespan_s": p_span, "p50_ms": q(p_lat, 50),
                      "p99_ms": q(p_lat, 99), "gpu_util_mean": clk_p.summary().get("util_mean"),
                      "kernel_s_sum": p_kernel, "host_s_sum": p_host},
            "batched": {"configs_per_s": configs / b_span, "makespan_s": b_span,
                        "gpu_util_mean": clk_b.summary().get("util_mean"),
                        "note": "one sqsg_optimize_batch call over all jobs, no arrivals"},
            "served_over_plain": p_span / s_span,
            "bound": {"kernel_s_sum_alone": p_kernel,
                      "plain_over_kernel_sum": p_span / p_kernel if p_kernel else None,
                      "note": "kernel_s_sum_alone is the summed engine-kernel time of the jobs run one at a time; "
                              "a served makespan cannot fall much below it when large jobs fill the GPU alone, so "
                              "plain_over_kernel_sum bounds served/plain for this mix"},
            "parity": {"served_identical_to_plain": same, "batched_identical_to_plain": same_b, "jobs": n_jobs},
            "e2e": {"value": value, "unit": "configs/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
            "roofline": {"bound": "smem", "achieved": achieved, "peak": smem_bw / 1e9, "unit": "GB/s",
                         "frac": achieved / (smem_bw / 1e9), "traffic": None,
                         "algorithmic": "2*P bytes of shared-memory species reads per configuration, summed over jobs",
                         "peak_source": "measured in this run: conflict-free LDS.32 microbenchmark"},
            "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": s_stats["launches"]}


def run_served(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    line = served_measure(args, local, world, rank)
    if line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="systematic",
                    choices=["systematic", "random", "quinary", "split", "split_single", "fcc500", "served"])
    ap.add_argument("--jobs", type=int, default=200, help="served: jobs in the stream")
    ap.add_argument("--rate", type=float, default=200.0, help="served: Poisson arrival rate, jobs/s")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-seconds", type=float, default=4.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="only the headline workload (by default the run adds the random, quinary, split and served "
                         "workloads, once each, on one GPU)")
    ap.add_argument("--limit", type=int, default=0, help="evaluate only the first LIMIT ranks (profiling)")
    ap.add_argument("--max-results", type=int, default=1 << 16,
                    help="record capacity per step; the exact objective levels do not depend on it")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "served":
        run_served(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
