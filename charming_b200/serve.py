"""Jacobi2d solve server through the C ABI (charming_serve_*).

One long-lived scheduler launch holds a pool of worker chares; requests
submitted while others run are admitted into it as request slots, workers
and HBM (under a byte budget) free up, and their chares share the PEs with
the requests already running (continuous batching). Results stay resident
until released; ``fetch`` copies one out while the server keeps running.

While a server runs it holds every PE: no other program of the library can
run, and nothing may synchronise the whole device (the launch only ends at
``stop``).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check
from .jacobi import Problem
from .runtime import runtime


@dataclass
class Completion:
    tag: int
    status: int
    sweeps: int
    res0: float
    res_last: float
    submit_s: float
    admit_s: float
    done_s: float

    @property
    def latency_s(self) -> float:
        return self.done_s - self.submit_s


class Server:
    def __init__(self, hbm_budget_bytes: int, max_inflight: int = 256, workers_per_pe: int = 16,
                 chare_side: int = 2048, dtype: str = "f32", deadline_s: float = 600.0):
        self.rt = runtime()
        self.lib = self.rt.lib
        self.dtype = np.float64 if dtype in ("f64", "float64", np.float64) else np.float32
        cfg = _lib.ServeConfig()
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.max_inflight = max_inflight
        cfg.workers_per_pe = workers_per_pe
        cfg.chare_side = chare_side
        cfg.dtype = _lib.F64 if self.dtype == np.float64 else _lib.F32
        cfg.deadline_s = deadline_s
        h = C.c_void_p()
        check(self.lib.charming_serve_start(C.byref(cfg), C.byref(h)), "charming_serve_start")
        self.h = h
        self.problems: dict[int, Problem] = {}
        self._buf = (_lib.ServeCompletion * 512)()

    def submit(self, problem: Problem, tag: int) -> None:
        p = problem.to_c()
        check(self.lib.charming_serve_submit(self.h, C.byref(p), C.c_uint64(tag)), "charming_serve_submit")
        self.problems[tag] = problem

    def poll(self) -> list[Completion]:
        n = C.c_int(0)
        check(self.lib.charming_serve_poll(self.h, self._buf, len(self._buf), C.byref(n)),
              "charming_serve_poll")
        return [Completion(c.tag, c.status, c.sweeps, c.res0, c.res_last, c.submit_s, c.admit_s,
                           c.done_s) for c in self._buf[: n.value]]

    def wait(self, tags, timeout_s: float = 60.0) -> dict[int, Completion]:
        """Polls until every tag in `tags` completed."""
        want, got = set(tags), {}
        t_end = time.monotonic() + timeout_s
        while want - got.keys():
            for c in self.poll():
                got[c.tag] = c
            if time.monotonic() > t_end:
                raise TimeoutError(f"requests {sorted(want - got.keys())[:8]} not done")
            time.sleep(0.0002)
        return got

    def fetch(self, tag: int, out: np.ndarray | None = None) -> np.ndarray:
        p = self.problems[tag]
        if out is None:
            out = np.empty((p.ny + 2, p.nx + 2), dtype=self.dtype)
        assert out.dtype == self.dtype and out.shape == (p.ny + 2, p.nx + 2) and out.flags.c_contiguous
        check(self.lib.charming_serve_fetch(self.h, C.c_uint64(tag), out.ctypes.data), "charming_serve_fetch")
        return out

    def release(self, tag: int) -> None:
        check(self.lib.charming_serve_release(self.h, C.c_uint64(tag)), "charming_serve_release")
        self.problems.pop(tag, None)

    def stop(self) -> dict:
        if not self.h:
            return {}
        st = _lib.ServeStats()
        rc = self.lib.charming_serve_stop(self.h, C.byref(st))
        self.h = None
        check(rc, "charming_serve_stop")
        return {f: getattr(st, f) for f, _ in _lib.ServeStats._fields_}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if self.h:
            try:
                self.stop()
            except Exception:
                if exc[0] is None:
                    raise
