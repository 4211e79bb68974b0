"""Host-side logic of the native library without a GPU: launch plans (which evaluation path a job
takes), process-wide options, and the per-device bookkeeping of the dynamic shared-memory attribute."""
import os
import subprocess

import pytest

import cases
import sqsgenerator_b200 as S
from sqsgenerator_b200 import _native as N
from sqsgenerator_b200.optimize import build_job

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def plan_of(cfg):
    c = S.parse_config(cfg)
    d = S.prepare(c)
    job, bufs = build_job(c, d)
    return N.plan(job)


def test_plan_paths_without_a_device():
    p = plan_of(cases.fcc32("double"))
    assert p["kernel"] == "sqsg_engine_mask" and p["parts"][0]["path"] == "bitmask"
    p = plan_of(cases.quinary("double", cells=(4, 4, 4)))
    assert p["kernel"] == "sqsg_engine_lat5" and p["parts"][0]["path"] == "lattice"
    p = plan_of(cases.rocksalt_split("double", cells=(3, 3, 3)))
    assert p["kernel"] == "sqsg_engine_lat2" and [x["path"] for x in p["parts"]] == ["lattice", "lattice"]
    with N.options(force_general=1):
        p = plan_of(cases.quinary("double", cells=(4, 4, 4)))
        assert p["kernel"] == "sqsg_engine_wide" and p["parts"][0]["path"] == "general"
        assert p["parts"][0]["stream_narrow"]
        p = plan_of(cases.rocksalt_split("double", cells=(3, 3, 3)))
        assert [x["path"] for x in p["parts"]] == ["general", "general"]
        assert not any(x["stream_staged"] for x in p["parts"])  # split jobs read the stream through L1


def _job(cfg, **kw):
    c = S.parse_config(cfg)
    d = S.prepare(c)
    return c, d, build_job(c, d, **kw)


def test_lattice_hint_is_checked():
    """The supercell hint only selects the lattice path when it is consistent with the pair list."""
    cfg = cases.quinary("double", cells=(3, 3, 3))
    c, d, (job, bufs) = _job(cfg, lattice_hint=False)
    assert N.plan(job)["parts"][0]["path"] == "general"
    # a hint that swaps two sites' cells: some translation classes become incomplete
    bad = d[0].lattice.copy()
    bad[[0, 5], 1:] = bad[[5, 0], 1:]
    d[0].lattice = bad
    job, bufs = build_job(c, d)
    assert N.plan(job)["parts"][0]["path"] == "general"
    # a cell index out of range is rejected too
    c, d, _ = _job(cfg)
    d[0].lattice = d[0].lattice.copy()
    d[0].lattice[3, 2] = 99
    job, bufs = build_job(c, d)
    assert N.plan(job)["parts"][0]["path"] == "general"


def test_lattice_hint_up_to_128_cells():
    """Cell sets of two words: 125 cells take sqsg_engine_latw up to five species; six species or more
    than 128 cells take the pair stream."""
    cfg = cases.fcc32("double", composition={"Ti": 250, "Al": 250}, iterations=1000)
    cfg["structure"]["supercell"] = [5, 5, 5]
    c, d, (job, bufs) = _job(cfg)
    with N.options(use_tuning=0):  # the rules' path (a tuning table may prefer the pair stream)
        p = N.plan(job)
    assert p["parts"][0]["path"] == "lattice" and p["kernel"] == "sqsg_engine_latw"
    cfg6 = cases.fcc32("double", composition={e: 500 // 6 + (1 if k < 500 % 6 else 0)
                                              for k, e in enumerate(("Ti", "Al", "Nb", "V", "Zr", "Hf"))},
                       iterations=1000)
    cfg6["structure"]["supercell"] = [5, 5, 5]
    c, d, (job, bufs) = _job(cfg6)
    assert N.plan(job)["parts"][0]["path"] == "general"
    cfg216 = cases.fcc32("double", composition={"Ti": 432, "Al": 432}, iterations=1000)
    cfg216["structure"]["supercell"] = [6, 6, 6]
    c, d, (job, bufs) = _job(cfg216)
    assert N.plan(job)["parts"][0]["path"] == "general"


def test_force_general_option():
    with N.options(force_general=1):
        assert N.get_option("force_general") == 1
        assert plan_of(cases.fcc32("double"))["parts"][0]["path"] == "general"
    assert N.get_option("force_general") == 0
    assert plan_of(cases.fcc32("double"))["parts"][0]["path"] == "bitmask"


def test_option_errors():
    with pytest.raises(N.NativeError) as e:
        N.set_option("no_such_option", 1)
    assert e.value.status_name == "SQSG_ERR_INVALID_ARGUMENT"
    with pytest.raises(N.NativeError) as e:
        N.set_option("stage_wait_ns", 0)
    assert e.value.status_name == "SQSG_ERR_OUT_OF_RANGE"
    assert N.get_option("stage_wait_ns") == 2_000_000_000


def test_plan_validates_like_optimize():
    with pytest.raises(N.NativeError) as e:
        plan_of(cases.fcc32("double", keep=4000))
    assert e.value.status_name == "SQSG_ERR_UNSUPPORTED"


TRACKER_TEST = r"""
#include <cstdio>
#include <vector>
#include "attr_tracker.h"
int main() {
  sqsg::DynamicSmemTracker t;
  std::vector<std::pair<int, size_t>> calls;  // (device, bytes) of every attribute write
  int dev = 0;
  auto set = [&](size_t b) { calls.push_back({dev, b}); return 0; };
  static int k1, k2;
  dev = 0; if (t.raise(0, &k1, 100000, set)) return 1;
  dev = 1; if (t.raise(1, &k1, 50000, set)) return 2;   // another device: must be set there too
  dev = 0; if (t.raise(0, &k1, 80000, set)) return 3;   // below what device 0 has: no write
  dev = 0; if (t.raise(0, &k2, 80000, set)) return 4;   // another kernel: its own record
  dev = 1; if (t.raise(1, &k1, 120000, set)) return 5;  // raised on device 1 only
  int fail_dev = 0;
  auto failing = [&](size_t) { fail_dev = 1; return 7; };
  if (t.raise(0, &k1, 200000, failing) != 7) return 6;  // a failed write leaves the record alone
  if (t.current(0, &k1) != 100000 || t.current(1, &k1) != 120000 || t.current(0, &k2) != 80000) return 8;
  const std::vector<std::pair<int, size_t>> want = {{0, 100000}, {1, 50000}, {0, 80000}, {1, 120000}};
  if (calls != want) return 9;
  std::printf("ok\n");
  return 0;
}
"""


def test_dynamic_smem_tracker_is_per_device(tmp_path):
    """A process that launches on two devices must raise the attribute on each: the bookkeeping keeps
    one record per (device, kernel) and only raises it (compiled here with g++ and a fake setter)."""
    src = tmp_path / "tracker_test.cpp"
    src.write_text(TRACKER_TEST)
    exe = tmp_path / "tracker_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "sqsgenerator_b200", "csrc"), str(src),
                    "-o", str(exe), "-pthread"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", (out.returncode, out.stdout, out.stderr)


def test_tuning_option_and_bucket():
    c, d, (job, bufs) = _job(cases.quinary("double", cells=(4, 4, 4)))
    p = N.plan(job)
    assert p["bucket"] > 0 and p["bucket"] == N.plan(job)["bucket"]
    assert N.get_option("use_tuning") == 1
    with N.options(use_tuning=0):
        assert not N.plan(job)["tuned"]
    # another shape, another bucket
    c2, d2, (job2, bufs2) = _job(cases.quinary("double", cells=(3, 3, 3)))
    assert N.plan(job2)["bucket"] != p["bucket"]


def test_candidate_budget_options():
    assert N.get_option("default_candidates") == 1 << 20
    assert N.get_option("rerun_record_bytes") == 4 << 30
    with N.options(default_candidates=4096, rerun_record_bytes=1 << 24):
        assert N.get_option("default_candidates") == 4096
        assert N.get_option("rerun_record_bytes") == 1 << 24
    assert N.get_option("default_candidates") == 1 << 20
    for name in ("default_candidates", "rerun_record_bytes"):
        with pytest.raises(N.NativeError):
            N.set_option(name, 0)


def test_rapidrand_debug_option_takes_the_pair_stream():
    """The reference-stream debug mode runs on the pair-stream path (its chains need the species
    columns); without it the same job takes the bit-mask path."""
    assert N.get_option("rapidrand") == 0
    cfg = cases.fcc32("double", iterations=5000, chunk_size=1000)
    assert plan_of(cfg)["parts"][0]["path"] == "bitmask"
    with N.options(rapidrand=1):
        assert plan_of(cfg)["parts"][0]["path"] == "general"
    assert N.get_option("rapidrand") == 0


def test_binary_floyd_option_sets_the_draws_per_configuration():
    """A random window of two species draws the sites of its rarer species (Floyd's sampling); with
    binary_floyd = 0, or with three species, a window takes n - 1 Fisher-Yates draws; systematic jobs
    draw nothing."""
    assert N.get_option("binary_floyd") == 1
    assert plan_of(cases.fcc32("double", iterations=1000))["shuffle_draws"] == 16
    assert plan_of(cases.fcc32("double", composition={"Ti": 7, "Al": 25}, iterations=1000))["shuffle_draws"] == 7
    assert plan_of(cases.fcc32("double", composition={"Ti": 11, "Al": 11, "Nb": 10},
                               iterations=1000))["shuffle_draws"] == 31
    assert plan_of(cases.rocksalt_split("double", iterations=1000))["shuffle_draws"] == 16 + 4  # Ti16Al16, N28B4
    assert plan_of(cases.fcc32("double", iteration_mode="systematic", seed=None,
                               iterations=None))["shuffle_draws"] == 0
    with N.options(binary_floyd=0):
        assert plan_of(cases.fcc32("double", iterations=1000))["shuffle_draws"] == 31
        assert plan_of(cases.rocksalt_split("double", iterations=1000))["shuffle_draws"] == 31 + 31
    with N.options(rapidrand=1):  # the reference's stream: Fisher-Yates on every window
        assert plan_of(cases.fcc32("double", iterations=1000, chunk_size=100))["shuffle_draws"] == 31
