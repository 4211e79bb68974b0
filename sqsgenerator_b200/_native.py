"""ctypes binding of ``libsqsg_b200.so`` (declared in ``include/sqsgen_b200.h``).

The library is built in-tree (``sqsgenerator_b200/build.py``). Importing this module never falls
back to another implementation: when the shared library is missing, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libsqsg_b200.so")

SQSG_OK = 0
STATUS_NAMES = {
    0: "SQSG_OK",
    1: "SQSG_ERR_INVALID_ARGUMENT",
    2: "SQSG_ERR_OUT_OF_RANGE",
    3: "SQSG_ERR_CAPACITY",
    4: "SQSG_ERR_CUDA",
    5: "SQSG_ERR_UNSUPPORTED",
    6: "SQSG_ERR_TIMEOUT",
    7: "SQSG_ERR_BUSY",
}

#: Every entry point the header declares (checked by the CPU test-suite).
EXPORTED = (
    "sqsg_version", "sqsg_last_error", "sqsg_device_count",
    "sqsg_supercell", "sqsg_distance_matrix", "sqsg_shell_matrix", "sqsg_distances_naive",
    "sqsg_distances_histogram", "sqsg_prefactors", "sqsg_pairs", "sqsg_sort_by_sublattice",
    "sqsg_num_permutations", "sqsg_rank_permutation", "sqsg_unrank_permutation",
    "sqsg_optimize", "sqsg_run_count", "sqsg_run_copy", "sqsg_run_statistics", "sqsg_run_free",
    "sqsg_optimize_trace", "sqsg_optimize_batch", "sqsg_run_levels", "sqsg_run_info",
    "sqsg_microbench", "sqsg_run_transfer", "sqsg_optimize_levels_noalloc",
    "sqsg_server_create", "sqsg_server_submit", "sqsg_server_wait", "sqsg_server_stats", "sqsg_server_destroy",
    "sqsg_server_running", "sqsg_set_option", "sqsg_get_option", "sqsg_plan_job", "sqsg_run_stages", "sqsg_autotune",
)

PATH_NAMES = {0: "general", 1: "bitmask", 2: "lattice"}


class NativeError(RuntimeError):
    """A non-OK sqsg_status, with the library's message."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.status_name}: {message}")


class SqsgSublattice(C.Structure):
    _fields_ = [
        ("n_sites", C.c_uint32),
        ("n_species", C.c_uint32),
        ("n_shells", C.c_uint32),
        ("n_pairs", C.c_uint32),
        ("n_windows", C.c_uint32),
        ("reserved", C.c_uint32),
        ("pairs", C.c_void_p),
        ("species", C.c_void_p),
        ("windows", C.c_void_p),
        ("prefactors", C.c_void_p),
        ("pair_weights", C.c_void_p),
        ("target", C.c_void_p),
        ("lattice", C.c_void_p),
        ("cells", C.c_uint32 * 3),
        ("n_basis", C.c_uint32),
    ]


class SqsgStatistics(C.Structure):
    _fields_ = [
        ("finished", C.c_uint64),
        ("working", C.c_uint64),
        ("best_rank", C.c_uint64),
        ("best_objective", C.c_double),
        ("timings_ns", C.c_uint64 * 4),
    ]


CALLBACK = C.CFUNCTYPE(C.c_int, C.POINTER(SqsgStatistics), C.c_void_p)


class SqsgJob(C.Structure):
    _fields_ = [
        ("prec", C.c_int32),
        ("iteration_mode", C.c_int32),
        ("sublattice_mode", C.c_int32),
        ("n_sublattices", C.c_uint32),
        ("sublattices", C.c_void_p),
        ("iterations", C.c_uint64),
        ("chunk_size", C.c_uint64),
        ("keep", C.c_uint64),
        ("max_results_per_objective", C.c_int64),
        ("seed", C.c_uint64),
        ("has_seed", C.c_int32),
        ("device", C.c_int32),
        ("cancel", C.c_void_p),
        ("callback", CALLBACK),
        ("user", C.c_void_p),
        ("max_results", C.c_uint64),
        ("range_first", C.c_uint64),
        ("range_count", C.c_uint64),
    ]


class SqsgPartPlan(C.Structure):
    _fields_ = [("path", C.c_int32), ("stream_narrow", C.c_int32), ("stream_staged", C.c_int32),
                ("lattice_units", C.c_uint32)]


class SqsgPlan(C.Structure):
    _fields_ = [("n_parts", C.c_uint32), ("smem_bytes", C.c_uint32), ("ctas_per_sm", C.c_uint32),
                ("record_bytes", C.c_uint32), ("kernel", C.c_char * 32), ("parts", SqsgPartPlan * 8),
                ("bucket", C.c_uint64), ("tuned", C.c_int32), ("shuffle_draws", C.c_uint32)]


class SqsgTuning(C.Structure):
    _fields_ = [("path", C.c_int32), ("stream_staged", C.c_int32), ("ctas_per_sm", C.c_uint32),
                ("tile_cap", C.c_uint32), ("configs_per_s", C.c_double)]


class SqsgServerOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("max_jobs", C.c_uint32),
        ("arena_bytes", C.c_uint64),
        ("default_max_results", C.c_uint64),
    ]


class SqsgServerCounters(C.Structure):
    _fields_ = [(name, C.c_uint64) for name in ("submitted", "admitted", "completed", "pending", "active",
                                                  "configurations", "launches", "arena_free_bytes")]


_LIB = None
_LOCK = threading.Lock()


def lib():
    """Load the native library (raises when it has not been built)."""
    global _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python sqsgenerator_b200/build.py` "
                "(there is no CPU fallback)"
            )
        L = C.CDLL(LIB_PATH)
        L.sqsg_version.restype = C.c_char_p
        L.sqsg_last_error.restype = C.c_size_t
        L.sqsg_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.sqsg_device_count.restype = C.c_int
        vp, u32, u64, dbl = C.c_void_p, C.c_uint32, C.c_uint64, C.c_double
        L.sqsg_supercell.argtypes = [C.c_int, vp, vp, vp, u32, u32, u32, u32, vp, vp, vp]
        L.sqsg_distance_matrix.argtypes = [C.c_int, vp, vp, u32, vp]
        L.sqsg_shell_matrix.argtypes = [C.c_int, vp, u32, vp, u32, dbl, dbl, vp]
        L.sqsg_distances_naive.argtypes = [C.c_int, vp, u32, dbl, dbl, vp, C.POINTER(u32)]
        L.sqsg_distances_histogram.argtypes = [C.c_int, vp, u32, dbl, dbl, vp, C.POINTER(u32)]
        L.sqsg_prefactors.argtypes = [C.c_int, vp, u32, vp, u32, vp, vp]
        L.sqsg_pairs.argtypes = [vp, u32, vp, u32, vp, C.POINTER(u32)]
        L.sqsg_sort_by_sublattice.argtypes = [vp, u32, u32, vp, vp, C.POINTER(u32)]
        L.sqsg_num_permutations.argtypes = [vp, u32, C.POINTER(u64)]
        L.sqsg_rank_permutation.argtypes = [vp, u32, C.POINTER(u64)]
        L.sqsg_unrank_permutation.argtypes = [vp, u32, u64]
        L.sqsg_optimize.argtypes = [C.POINTER(SqsgJob), C.POINTER(vp)]
        L.sqsg_optimize_batch.argtypes = [C.POINTER(SqsgJob), u32, C.POINTER(vp)]
        L.sqsg_optimize_trace.argtypes = [C.POINTER(SqsgJob), C.POINTER(vp), u64, C.POINTER(u64), vp, vp, vp, vp]
        L.sqsg_run_count.restype = u64
        L.sqsg_run_count.argtypes = [vp]
        L.sqsg_run_copy.argtypes = [vp, u64, u64, vp, vp, vp, vp, vp]
        L.sqsg_run_statistics.argtypes = [vp, C.POINTER(SqsgStatistics)]
        L.sqsg_run_free.argtypes = [vp]
        L.sqsg_run_levels.argtypes = [vp, C.POINTER(u32), vp, vp, vp]
        L.sqsg_run_info.argtypes = [vp, C.POINTER(u64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.sqsg_run_transfer.argtypes = [vp, C.POINTER(u64), C.POINTER(u64)]
        L.sqsg_run_stages.argtypes = [vp, vp, C.POINTER(u32)]
        L.sqsg_autotune.argtypes = [C.POINTER(SqsgJob), dbl, C.POINTER(SqsgTuning), C.POINTER(SqsgTuning),
                                    C.POINTER(u32)]
        L.sqsg_optimize_levels_noalloc.argtypes = [C.POINTER(SqsgJob), vp, C.POINTER(u32), vp, vp, vp,
                                                   C.POINTER(SqsgStatistics), C.c_char_p, C.c_size_t]
        L.sqsg_server_create.argtypes = [C.POINTER(SqsgServerOptions), C.POINTER(vp)]
        L.sqsg_server_submit.argtypes = [vp, C.POINTER(SqsgJob), C.POINTER(u64)]
        L.sqsg_server_wait.argtypes = [vp, u64, C.c_int64, C.POINTER(vp)]
        L.sqsg_server_stats.argtypes = [vp, C.POINTER(SqsgServerCounters)]
        L.sqsg_server_destroy.argtypes = [vp]
        L.sqsg_server_running.argtypes = [vp, C.POINTER(u32)]
        L.sqsg_set_option.argtypes = [C.c_char_p, C.c_int64]
        L.sqsg_get_option.argtypes = [C.c_char_p, C.POINTER(C.c_int64)]
        L.sqsg_plan_job.argtypes = [C.POINTER(SqsgJob), C.POINTER(SqsgPlan)]
        L.sqsg_microbench.argtypes = [C.c_int, C.c_int, C.POINTER(dbl), C.POINTER(dbl)]
        for name in EXPORTED:
            if name not in ("sqsg_version", "sqsg_last_error", "sqsg_device_count", "sqsg_run_count",
                            "sqsg_run_free"):
                getattr(L, name).restype = C.c_int
        _LIB = L
        return _LIB


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().sqsg_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != SQSG_OK:
        raise NativeError(status, last_error())


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def prec_code(dtype) -> int:
    return 1 if np.dtype(dtype) == np.float64 else 0


def set_option(name: str, value: int) -> None:
    check(lib().sqsg_set_option(name.encode(), int(value)))


def get_option(name: str) -> int:
    v = C.c_int64()
    check(lib().sqsg_get_option(name.encode(), C.byref(v)))
    return int(v.value)


class options:
    """Context manager that sets process-wide library options and restores them on exit."""

    def __init__(self, **values):
        self.values = values
        self.saved = {}

    def __enter__(self):
        for k, v in self.values.items():
            self.saved[k] = get_option(k)
            set_option(k, v)
        return self

    def __exit__(self, *exc):
        for k, v in self.saved.items():
            set_option(k, v)


def plan(job) -> dict:
    """sqsg_plan_job of a native job: kernel, shared memory, CTAs per SM and each part's path."""
    p = SqsgPlan()
    check(lib().sqsg_plan_job(C.byref(job), C.byref(p)))
    parts = [dict(path=PATH_NAMES.get(p.parts[k].path, str(p.parts[k].path)),
                  stream_narrow=bool(p.parts[k].stream_narrow), stream_staged=bool(p.parts[k].stream_staged),
                  lattice_units=int(p.parts[k].lattice_units))
             for k in range(p.n_parts)]
    return dict(kernel=p.kernel.decode(), smem_bytes=int(p.smem_bytes), ctas_per_sm=int(p.ctas_per_sm),
                record_bytes=int(p.record_bytes), parts=parts, bucket=int(p.bucket), tuned=bool(p.tuned),
                shuffle_draws=int(p.shuffle_draws))


def autotune(job, seconds: float = 2.0) -> tuple[dict, list[dict]]:
    """sqsg_autotune of a native job: (chosen, every choice measured)."""
    best = SqsgTuning()
    tried = (SqsgTuning * 64)()
    n = C.c_uint32(64)
    check(lib().sqsg_autotune(C.byref(job), float(seconds), C.byref(best), tried, C.byref(n)))
    conv = lambda t: dict(path=PATH_NAMES.get(t.path, str(t.path)), stream_staged=int(t.stream_staged),  # noqa: E731
                          ctas_per_sm=int(t.ctas_per_sm), tile_cap=int(t.tile_cap),
                          configs_per_s=float(t.configs_per_s))
    return conv(best), [conv(tried[k]) for k in range(min(n.value, 64))]


STAGE_NAMES = ("prepare", "upload", "kernel", "wait", "levels", "select", "total")


def run_stages(run) -> dict:
    """Host time (seconds) per stage of the sqsg_optimize call that produced `run`."""
    ns = np.zeros(len(STAGE_NAMES), np.uint64)
    n = C.c_uint32(len(STAGE_NAMES))
    check(lib().sqsg_run_stages(run, ptr(ns), C.byref(n)))
    return {name: float(ns[k]) * 1e-9 for k, name in enumerate(STAGE_NAMES[: n.value])}


def device_count() -> int:
    return int(lib().sqsg_device_count())


def version() -> str:
    return lib().sqsg_version().decode()


# ----------------------------------------------------------------------------- geometry wrappers
def supercell(lattice, frac, species, a, b, c, dtype=np.float64):
    lattice = np.ascontiguousarray(lattice, dtype=dtype)
    frac = np.ascontiguousarray(frac, dtype=dtype)
    species = np.ascontiguousarray(species, dtype=np.uint8)
    n = len(species)
    m = n * a * b * c
    lo = np.zeros((3, 3), dtype=dtype)
    fo = np.zeros((m, 3), dtype=dtype)
    so = np.zeros(m, dtype=np.uint8)
    check(lib().sqsg_supercell(prec_code(dtype), ptr(lattice), ptr(frac), ptr(species), n, a, b, c,
                               ptr(lo), ptr(fo), ptr(so)))
    return lo, fo, so


def distance_matrix(lattice, frac, dtype=np.float64):
    lattice = np.ascontiguousarray(lattice, dtype=dtype)
    frac = np.ascontiguousarray(frac, dtype=dtype)
    n = frac.shape[0]
    out = np.zeros((n, n), dtype=dtype)
    check(lib().sqsg_distance_matrix(prec_code(dtype), ptr(lattice), ptr(frac), n, ptr(out)))
    return out


def shell_matrix(dist, radii, atol, rtol):
    dist = np.ascontiguousarray(dist)
    radii = np.ascontiguousarray(radii, dtype=dist.dtype)
    n = dist.shape[0]
    out = np.zeros((n, n), dtype=np.uint32)
    check(lib().sqsg_shell_matrix(prec_code(dist.dtype), ptr(dist), n, ptr(radii), len(radii), float(atol),
                                  float(rtol), ptr(out)))
    return out


def _radii(fn, dist, a, b):
    dist = np.ascontiguousarray(dist)
    n = dist.shape[0]
    cap = C.c_uint32(max(16, n * n + 1))
    out = np.zeros(cap.value, dtype=dist.dtype)
    check(fn(prec_code(dist.dtype), ptr(dist), n, float(a), float(b), ptr(out), C.byref(cap)))
    return out[: cap.value].copy()


def distances_naive(dist, atol, rtol):
    return _radii(lib().sqsg_distances_naive, dist, atol, rtol)


def distances_histogram(dist, bin_width, peak_isolation):
    return _radii(lib().sqsg_distances_histogram, dist, bin_width, peak_isolation)


def prefactors(shells, shell_ids, species, dtype=np.float64):
    shells = np.ascontiguousarray(shells, dtype=np.uint32)
    ids = np.ascontiguousarray(sorted(shell_ids), dtype=np.uint32)
    species = np.ascontiguousarray(species, dtype=np.uint8)
    K = len(set(species.tolist()))
    out = np.zeros((len(ids), K, K), dtype=dtype)
    check(lib().sqsg_prefactors(prec_code(dtype), ptr(shells), shells.shape[0], ptr(ids), len(ids),
                                ptr(species), ptr(out)))
    return out


def pairs(shells, shell_ids):
    shells = np.ascontiguousarray(shells, dtype=np.uint32)
    ids = np.ascontiguousarray(sorted(shell_ids), dtype=np.uint32)
    n = shells.shape[0]
    cnt = C.c_uint32(0)
    check_cap = lib().sqsg_pairs(ptr(shells), n, ptr(ids), len(ids), None, C.byref(cnt))
    if check_cap not in (SQSG_OK, 3):
        check(check_cap)
    out = np.zeros((max(cnt.value, 1), 3), dtype=np.uint32)
    cap = C.c_uint32(cnt.value)
    check(lib().sqsg_pairs(ptr(shells), n, ptr(ids), len(ids), ptr(out), C.byref(cap)))
    return out[: cap.value]


def sort_by_sublattice(sublattice_of_site, n_sublattices):
    s = np.ascontiguousarray(sublattice_of_site, dtype=np.uint32)
    n = len(s)
    order = np.zeros(n, dtype=np.uint32)
    windows = np.zeros((max(n_sublattices, 1) + 1, 2), dtype=np.uint32)
    nw = C.c_uint32(windows.shape[0])
    check(lib().sqsg_sort_by_sublattice(ptr(s), n, n_sublattices, ptr(order), ptr(windows), C.byref(nw)))
    return order, windows[: nw.value].copy()


def num_permutations(conf):
    c = np.ascontiguousarray(conf, dtype=np.uint8)
    out = C.c_uint64(0)
    check(lib().sqsg_num_permutations(ptr(c), len(c), C.byref(out)))
    return int(out.value)


def rank_permutation(conf):
    c = np.ascontiguousarray(conf, dtype=np.uint8)
    out = C.c_uint64(0)
    check(lib().sqsg_rank_permutation(ptr(c), len(c), C.byref(out)))
    return int(out.value)


def unrank_permutation(conf, rank):
    c = np.ascontiguousarray(conf, dtype=np.uint8).copy()
    check(lib().sqsg_unrank_permutation(ptr(c), len(c), int(rank)))
    return c


def microbench(kind: int, device: int = 0):
    """(rate, seconds) of the shared-memory (kind 0, bytes/s), INT32 (kind 1, lane ops/s) or popcount
    (kind 2, 32-bit popcounts/s) microbenchmark."""
    r = C.c_double()
    t = C.c_double()
    check(lib().sqsg_microbench(kind, device, C.byref(r), C.byref(t)))
    return r.value, t.value
