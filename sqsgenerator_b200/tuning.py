"""The shipped tuning table: sqsg_autotune over representative job buckets, written as
``csrc/tuning_table.inc`` (compiled into the library).

A bucket is a job's shape (precision, mode, parts, largest species and shell counts, and the powers
of two of its sites and pairs; see ``bucket_key`` in ``csrc/prepare.cu``). For each representative
job below the autotuner times every launch choice that applies (evaluation path, pair-stream staging,
CTAs per SM, tile size) on short prefixes of the job and keeps the fastest. Run on the target GPU::

    python -m sqsgenerator_b200.tuning --seconds 1.5 --out sqsgenerator_b200/csrc/tuning_table.inc \\
        --report tuning_report.json

then rebuild the library. Results never depend on the table, only the speed.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import _native
from .config import parse_config
from .optimize import build_job, prepare

FCC = [[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]
BCC = [[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]]
ELEMENTS = ("Ti", "Al", "Nb", "V", "Zr")


def _cell(kind: str, rep: int, k: int, shells: int, prec: str = "double", iterations: int = 10_000_000):
    a, coords = (4.0, FCC) if kind == "fcc" else (2.87, BCC)
    n = len(coords) * rep ** 3
    counts = [n // k + (1 if i < n % k else 0) for i in range(k)]
    return dict(prec=prec, structure=dict(lattice=(np.eye(3) * a).tolist(), coords=coords, species=[1] * len(coords),
                                          supercell=[rep] * 3),
                composition=dict(zip(ELEMENTS, counts)), shell_weights={str(s): 1.0 / s for s in range(1, shells + 1)},
                iterations=iterations, seed=1, thread_config=1, keep=10)


def representative_jobs() -> dict:
    """The benchmark configurations' cells and the served stream's cell shapes."""
    jobs = {
        "fcc32_binary_2shells": _cell("fcc", 2, 2, 2, iterations=50_000_000),
        "fcc256_quinary_3shells": _cell("fcc", 4, 5, 3, iterations=20_000_000),
    }
    rocksalt = dict(prec="double", sublattice_mode="split",
                    structure=dict(lattice=(np.eye(3) * 4.2).tolist(),
                                   coords=FCC + [[0.5, 0.0, 0.0], [0.0, 0.5, 0.0], [0.0, 0.0, 0.5], [0.5, 0.5, 0.5]],
                                   species=[11] * 4 + [17] * 4, supercell=[3, 3, 3]),
                    composition=[{"sites": "Na", "Ti": 54, "Al": 54}, {"sites": "Cl", "N": 96, "B": 12}],
                    shell_weights=[{"1": 1.0, "2": 0.5}, {"1": 1.0, "2": 0.5}], iterations=100_000_000, seed=1,
                    thread_config=1)
    jobs["rocksalt216_split_double"] = rocksalt
    jobs["rocksalt216_split_single"] = dict(rocksalt, prec="single")
    for kind, rep in (("fcc", 2), ("bcc", 3), ("fcc", 3), ("bcc", 4), ("fcc", 4), ("fcc", 5)):
        for k in (2, 3, 5):
            for shells in (2, 4):
                jobs[f"{kind}{len(FCC if kind == 'fcc' else BCC) * rep ** 3}_k{k}_s{shells}"] = _cell(kind, rep, k, shells)
    return jobs


def summarize(report: dict) -> str:
    """Markdown table of a tuning report: per representative job the chosen launch choices, their rate, the
    rate of the fixed rules' choice (the path and stream staging `sqsg_plan_job` gives without the table, all
    CTAs that fit, tile cap 65536) and the spread of every measured choice. Needs no GPU."""
    rows = ["| representative job | bucket | chosen: path, staged, CTAs/SM, tile cap | configs/s | rules' choice configs/s "
            "| chosen / rules | choices | best / worst |", "|---|---:|---|---:|---:|---:|---:|---:|"]
    jobs = representative_jobs()
    prev = _native.get_option("use_tuning")
    _native.set_option("use_tuning", 0)
    try:
        for name, r in report.items():
            b, tried = r["best"], r["tried"]
            rules = None
            if name in jobs:
                c = parse_config(jobs[name])
                job, keep = build_job(c, prepare(c))
                part = _native.plan(job)["parts"][0]
                staged = int(part["stream_staged"]) if part["path"] == "general" else -1
                for t in tried:
                    if (t["path"] == part["path"] and t["ctas_per_sm"] == 0 and t["tile_cap"] == 65536
                            and (part["path"] != "general" or t["stream_staged"] == staged)):
                        rules = t["configs_per_s"]
                        break
            worst = min(t["configs_per_s"] for t in tried)
            rules_s = f"{rules / 1e6:.1f}e6" if rules else "—"
            ratio = f"{b['configs_per_s'] / rules:.2f}" if rules else "—"
            rows.append(f"| {name} | {r['bucket']} | {b['path']}, {b['stream_staged']}, {b['ctas_per_sm'] or 'all'}, "
                        f"{b['tile_cap']} | {b['configs_per_s'] / 1e6:.1f}e6 | {rules_s} | {ratio} | {len(tried)} | "
                        f"{b['configs_per_s'] / worst:.2f} |")
    finally:
        _native.set_option("use_tuning", prev)
    return "\n".join(rows) + "\n"


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--seconds", type=float, default=1.5, help="measuring budget per job")
    ap.add_argument("--out", default=None, help="path of the tuning_table.inc to write")
    ap.add_argument("--summarize", default=None, metavar="REPORT",
                    help="print the markdown summary of a report written by --report (no GPU needed) and exit")
    ap.add_argument("--report", default=None, help="JSON report of every measured choice")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    if args.summarize:
        with open(args.summarize) as f:
            print(summarize(json.load(f)), end="")
        return
    if not args.out:
        ap.error("--out is required when measuring")
    _native.set_option("use_tuning", 0)
    entries, report = {}, {}
    for name, cfg in representative_jobs().items():
        c = parse_config(cfg)
        d = prepare(c)
        job, keep = build_job(c, d, device=args.device)
        t0 = time.perf_counter()
        best, tried = _native.autotune(job, args.seconds)
        key = _native.plan(job)["bucket"]
        report[name] = dict(bucket=key, best=best, tried=tried, seconds=time.perf_counter() - t0)
        if key not in entries or best["configs_per_s"] > entries[key][1]["configs_per_s"]:
            entries[key] = (name, best)
        print(name, key, best, flush=True)
    lines = ["// Measured launch choices per job bucket: {bucket key, path, stage, CTAs per SM, tile cap}.",
             "// Written by sqsgenerator_b200/tuning.py from sqsg_autotune runs on a B200 (one line per bucket;",
             "// path 0 = the pair stream even where the lattice path applies, -1 = the rules' path)."]
    for key, (name, b) in sorted(entries.items()):
        path = 0 if b["path"] == "general" else -1
        lines.append(f"    {{{key}ull, {path}, {b['stream_staged']}, {b['ctas_per_sm']}u, {b['tile_cap']}u}},  // {name}")
    with open(args.out, "w") as f:
        f.write("\n".join(lines) + "\n")
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
