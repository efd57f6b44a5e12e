"""Jacobi2d chares through the C ABI (charming_jacobi2d_*).

Mirrors the reference's Jacobi example program (examples/jacobi2d/
jacobi2d.cu): a Dirichlet problem is decomposed into a px x py chare array,
chares exchange halos as messages every sweep, and the sweep is the
5-point average (c + l + r + u + d) * 0.2.  Grids are (ny+2) x (nx+2)
row-major arrays whose outer ring is the fixed boundary.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check
from .runtime import runtime


@dataclass
class Problem:
    nx: int
    ny: int
    max_sweeps: int
    px: int = 0
    py: int = 0
    check_every: int = 0
    tol: float = 0.0
    bc: tuple = (0.0, 0.0, 0.0, 0.0)  # top, bottom, left, right

    def to_c(self) -> _lib.JacobiProblem:
        p = _lib.JacobiProblem()
        p.nx, p.ny, p.px, p.py = self.nx, self.ny, self.px, self.py
        p.max_sweeps, p.check_every, p.tol = self.max_sweeps, self.check_every, self.tol
        for k in range(4):
            p.bc[k] = float(self.bc[k])
        return p


def reference_decomposition(n_chares: int, nx: int, ny: int) -> tuple[int, int]:
    """Surface-minimising split of n_chares into (cols, rows), the rule of
    examples/jacobi2d/jacobi2d.cu:37-57 (returns px = chares along x)."""
    best, rows, cols = 2.0 * (ny + nx), None, None
    for ipx in range(1, n_chares + 1):
        if n_chares % ipx == 0:
            ipy = n_chares // ipx
            surf = 2.0 * (ny / ipx + nx / ipy)
            if surf < best:
                best, rows, cols = surf, ipx, ipy
    if rows is None:
        raise ValueError(f"cannot decompose {n_chares} chares")
    return cols, rows


def initial_grid(nx: int, ny: int, bc, dtype=np.float64) -> np.ndarray:
    """The state charming_jacobi2d_init builds: ring from bc (top and bottom
    rows include the corners), interior 0."""
    g = np.zeros((ny + 2, nx + 2), dtype=dtype)
    g[:, 0] = bc[2]
    g[:, -1] = bc[3]
    g[0, :] = bc[0]
    g[-1, :] = bc[1]
    return g


@dataclass
class Result:
    sweeps: int
    checks: int
    res0: float
    res_last: float


class Jacobi2D:
    """A set of problems decomposed into chares, resident on the GPU."""

    def __init__(self, problems, dtype: str = "f64", chare_side: int = 0, tile_w: int = 0,
                 pipeline: bool = False, use_graph: bool = False, balance: bool = True,
                 halo_mode: int = 0, depth: int = 0):
        self.rt = runtime()
        self.lib = self.rt.lib
        self.problems = [p if isinstance(p, Problem) else Problem(**p) for p in problems]
        self.dtype = np.float64 if dtype in ("f64", "float64", np.float64) else np.float32
        arr = (_lib.JacobiProblem * len(self.problems))(*[p.to_c() for p in self.problems])
        opt = _lib.JacobiOptions()
        opt.dtype = _lib.F64 if self.dtype == np.float64 else _lib.F32
        opt.chare_side, opt.tile_w = chare_side, tile_w
        opt.pipeline, opt.use_graph, opt.balance = int(pipeline), int(use_graph), int(balance)
        opt.halo_mode = halo_mode
        opt.depth = depth
        h = C.c_void_p()
        check(self.lib.charming_jacobi2d_create(arr, len(self.problems), C.byref(opt), C.byref(h)),
              "charming_jacobi2d_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            self.lib.charming_jacobi2d_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self) -> None:
        check(self.lib.charming_jacobi2d_init(self.h), "charming_jacobi2d_init")

    def load(self, prob: int, grid: np.ndarray) -> None:
        p = self.problems[prob]
        g = np.ascontiguousarray(grid, dtype=self.dtype)
        assert g.shape == (p.ny + 2, p.nx + 2)
        check(self.lib.charming_jacobi2d_load(self.h, prob, g.ctypes.data), "charming_jacobi2d_load")

    def run(self) -> float:
        """One persistent launch that runs every problem to completion; returns
        its CUDA-event time in ms."""
        check(self.lib.charming_jacobi2d_run(self.h), "charming_jacobi2d_run")
        return self.info()["last_run_ms"]

    def run_n(self, n_runs: int) -> float:
        """n_runs runs enqueued back to back and synchronised once (no host
        work between them); returns the CUDA-event ms of all of them."""
        ms = C.c_double(0.0)
        check(self.lib.charming_jacobi2d_run_n(self.h, n_runs, C.byref(ms)), "charming_jacobi2d_run_n")
        return ms.value

    def store(self, prob: int, out: np.ndarray | None = None) -> np.ndarray:
        p = self.problems[prob]
        if out is None:
            out = np.empty((p.ny + 2, p.nx + 2), dtype=self.dtype)
        check(self.lib.charming_jacobi2d_store(self.h, prob, out.ctypes.data), "charming_jacobi2d_store")
        return out

    def solve_stream(self, prob: int, inputs, outputs) -> float:
        """Solves problem prob once per input grid, results into the matching
        output arrays, with the host copies of neighbouring solves
        overlapping each solve (pinned arrays overlap best); returns the ms
        from the first input copy to the last result copy."""
        p = self.problems[prob]
        ins = [np.ascontiguousarray(g, dtype=self.dtype) for g in inputs]
        for g, o in zip(ins, outputs):
            assert g.shape == o.shape == (p.ny + 2, p.nx + 2) and o.dtype == self.dtype and o.flags.c_contiguous
        n = len(ins)
        pin = (C.c_void_p * n)(*[g.ctypes.data for g in ins])
        pout = (C.c_void_p * n)(*[o.ctypes.data for o in outputs])
        ms = C.c_double(0.0)
        check(self.lib.charming_jacobi2d_solve_stream(self.h, prob, n, pin, pout, C.byref(ms)),
              "charming_jacobi2d_solve_stream")
        return ms.value

    def result(self, prob: int) -> Result:
        r = _lib.JacobiResult()
        check(self.lib.charming_jacobi2d_result(self.h, prob, C.byref(r)), "charming_jacobi2d_result")
        return Result(r.sweeps, r.checks, r.res0, r.res_last)

    def info(self) -> dict:
        i = _lib.JacobiInfo()
        check(self.lib.charming_jacobi2d_get_info(self.h, C.byref(i)), "charming_jacobi2d_get_info")
        return {f: getattr(i, f) for f, _ in _lib.JacobiInfo._fields_}
