"""ctypes front end of the C Jacobi oracle (liboracle_jacobi.so).
TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py; never by the product path."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from .msgmodel import mix64

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle_jacobi.so")
        if not os.path.exists(path):
            subprocess.run(["make"], cwd=HERE, check=True, capture_output=True)
        L = C.CDLL(path)
        dp, fp, i = C.POINTER(C.c_double), C.POINTER(C.c_float), C.c_int
        L.oracle_jacobi2d_f64.argtypes = [dp, i, i, i]
        L.oracle_jacobi2d_f64_omp.argtypes = [dp, i, i, i, i]
        L.oracle_jacobi2d_f32.argtypes = [fp, i, i, i, i]
        L.oracle_residual2_f64.argtypes = [dp, i, i]
        L.oracle_residual2_f64.restype = C.c_double
        L.oracle_residual2_f32.argtypes = [fp, i, i]
        L.oracle_residual2_f32.restype = C.c_double
        L.oracle_jacobi1d_f64.argtypes = [dp, i, i]
        L.oracle_decomp1d_f32.argtypes = [i, i, i, i, fp, fp]
        L.oracle_jacobi3d_f64.argtypes = [dp, i, i, i, i, i]
        _lib = L
    return _lib


def jacobi2d(grid: np.ndarray, sweeps: int, threads: int = 0) -> np.ndarray:
    """`sweeps` sweeps of the grid's dtype (serial when threads == 0)."""
    g = np.ascontiguousarray(grid).copy()
    ny, nx = g.shape[0] - 2, g.shape[1] - 2
    if g.dtype == np.float64:
        ptr = g.ctypes.data_as(C.POINTER(C.c_double))
        if threads:
            lib().oracle_jacobi2d_f64_omp(ptr, nx, ny, sweeps, threads)
        else:
            lib().oracle_jacobi2d_f64(ptr, nx, ny, sweeps)
    elif g.dtype == np.float32:
        lib().oracle_jacobi2d_f32(g.ctypes.data_as(C.POINTER(C.c_float)), nx, ny, sweeps,
                                  threads if threads else 1)
    else:
        raise TypeError(g.dtype)
    return g


def residual(grid: np.ndarray) -> float:
    """||S(u) - u||_2 with S evaluated in FP64."""
    g = np.ascontiguousarray(grid)
    ny, nx = g.shape[0] - 2, g.shape[1] - 2
    if g.dtype == np.float64:
        r2 = lib().oracle_residual2_f64(g.ctypes.data_as(C.POINTER(C.c_double)), nx, ny)
    else:
        r2 = lib().oracle_residual2_f32(g.ctypes.data_as(C.POINTER(C.c_float)), nx, ny)
    return float(np.sqrt(r2))


def jacobi1d(a: np.ndarray, width: int, sweeps: int) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float64).copy()
    lib().oracle_jacobi1d_f64(out.ctypes.data_as(C.POINTER(C.c_double)), width, sweeps)
    return out


def seeded_grid(nx: int, ny: int, seed: int) -> np.ndarray:
    """Grid of values (mix64(seed*2^32 + k) >> 11) * 2^-53 in [0, 1); the
    generator of oracle/ref/ref_jacobi_dump.cu."""
    k = np.arange((nx + 2) * (ny + 2), dtype=np.uint64)
    with np.errstate(over="ignore"):
        v = mix64((np.uint64(seed) << np.uint64(32)) + k) >> np.uint64(11)
    return (v.astype(np.float64) * (1.0 / 9007199254740992.0)).reshape(ny + 2, nx + 2)


def decomp1d_boundary(ny: int) -> np.ndarray:
    """Left/right column values of jacobi2d-decomp1d per global row g
    (examples/jacobi2d-decomp1d/jacobi2d.cu:424-433: sin(2*PI*(g-1)/(ny-3))
    with PI = 3.141592 as a float), float32[ny]."""
    pi = float(np.float32(3.141592))
    g = np.arange(ny, dtype=np.float64)
    return np.sin(2.0 * pi * (g - 1.0) / float(ny - 3)).astype(np.float32)


def decomp1d(n: int, nx: int, ny: int, iters: int) -> np.ndarray:
    """(ny-2) x nx float32 result of the decomp1d oracle."""
    bc = np.ascontiguousarray(decomp1d_boundary(ny))
    out = np.zeros((ny - 2, nx), dtype=np.float32)
    fp = C.POINTER(C.c_float)
    rc = lib().oracle_decomp1d_f32(n, nx, ny, iters, bc.ctypes.data_as(fp), out.ctypes.data_as(fp))
    if rc != 0:
        raise ValueError("decomp1d: sizes the decomposition does not cover")
    return out


def jacobi3d(grid: np.ndarray, sweeps: int, threads: int = 0) -> np.ndarray:
    """`sweeps` 7-point sweeps of an (nz+2, ny+2, nx+2) FP64 grid (x fastest,
    boundary shell fixed); serial when threads == 0."""
    g = np.ascontiguousarray(grid, dtype=np.float64).copy()
    nz, ny, nx = (d - 2 for d in g.shape)
    lib().oracle_jacobi3d_f64(g.ctypes.data_as(C.POINTER(C.c_double)), nx, ny, nz, sweeps, threads)
    return g


def seeded_grid3d(nx: int, ny: int, nz: int, seed: int) -> np.ndarray:
    """Every cell (shell included) = (mix64(seed * 2^32 + k) >> 11) * 2^-53,
    k the cell's linear index (the reference-kernel harness fills the same)."""
    k = np.arange((nx + 2) * (ny + 2) * (nz + 2), dtype=np.uint64)
    with np.errstate(over="ignore"):
        v = mix64((np.uint64(seed) << np.uint64(32)) + k)
    return ((v >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)).reshape(nz + 2, ny + 2, nx + 2)
