"""Served form: continuous batching of SQS jobs on one GPU (``sqsg_server_*`` in the C ABI).

Jobs submitted while others run are admitted as job slots and device memory free up and join the
persistent kernel that is already running; each result equals what ``optimize`` returns for the same
job. ``Server.result`` returns the reference-shaped ``SqsResultPack``.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import Any

from . import _native
from .config import parse_config
from .core import ParseError, SqsConfiguration
from .optimize import build_job, collect, prepare


class Server:
    def __init__(self, device: int = 0, *, arena_bytes: int = 0, max_jobs: int = 0, default_max_results: int = 0):
        opt = _native.SqsgServerOptions(device, max_jobs, arena_bytes, default_max_results)
        self._h = C.c_void_p()
        _native.check(_native.lib().sqsg_server_create(C.byref(opt), C.byref(self._h)))
        self.device = device
        self._jobs: dict[int, Any] = {}
        self._lock = threading.Lock()

    def submit(self, config: dict[str, Any] | SqsConfiguration | str, *, prepared=None) -> int:
        """Queue a job; returns its ticket. ``prepared`` may carry (config, data) from earlier."""
        if prepared is None:
            c = config if isinstance(config, SqsConfiguration) else parse_config(config)
            if isinstance(c, ParseError):
                raise ValueError(str(c))
            d = prepare(c)
        else:
            c, d = prepared
        job, bufs = build_job(c, d, device=self.device)
        ticket = C.c_uint64()
        _native.check(_native.lib().sqsg_server_submit(self._h, C.byref(job), C.byref(ticket)))
        with self._lock:
            self._jobs[ticket.value] = (c, d, bufs)
        return ticket.value

    def wait_run(self, ticket: int, timeout: float | None = None):
        """The raw native run handle of a finished job (free with sqsg_run_free)."""
        run = C.c_void_p()
        us = -1 if timeout is None else int(timeout * 1e6)
        _native.check(_native.lib().sqsg_server_wait(self._h, ticket, us, C.byref(run)))
        return run

    def result(self, ticket: int, timeout: float | None = None):
        run = self.wait_run(ticket, timeout)
        with self._lock:
            c, d, _ = self._jobs.pop(ticket)
        try:
            return collect(c, d, run)
        finally:
            _native.lib().sqsg_run_free(run)

    def stats(self) -> dict:
        st = _native.SqsgServerCounters()
        _native.check(_native.lib().sqsg_server_stats(self._h, C.byref(st)))
        return {name: int(getattr(st, name)) for name, _ in st._fields_}

    def close(self) -> None:
        if self._h:
            _native.lib().sqsg_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 — interpreter shutdown
            pass
