"""charming_jacobi2d_sweeps_noalloc: the Jacobi sweep entry point for callers
that must not allocate device memory (code that hands this library buffers
from its own pool and forbids allocations outside it, or that cannot pay
for the device synchronisation of a cudaMalloc). Its second grid lives in a
fixed 16 MiB scratch array inside the library, so its grids are limited to
(nx+2)*(ny+2)*element size <= 16 MiB.

The GPU tests compare it, bit for bit, with the chare entry point
(charming_jacobi2d_create/load/run/store) on two calls in a row with
different grids, so that scratch contents left by the first call would show
in the second. The test allocates the device grids itself (through torch):
only the entry point under test must not allocate.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from charming_b200 import _lib
from charming_b200.jacobi import Jacobi2D, Problem
from oracle.jacobi import jacobi2d, seeded_grid


def chare_result(grid, sweeps, dtype):
    """The existing entry point's grid after `sweeps` sweeps."""
    ny, nx = grid.shape[0] - 2, grid.shape[1] - 2
    with Jacobi2D([Problem(nx, ny, sweeps)], dtype=dtype) as j:
        j.load(0, grid)
        j.run()
        return j.store(0)


def noalloc_result(lib, torch, grid, sweeps, dtype):
    ny, nx = grid.shape[0] - 2, grid.shape[1] - 2
    d_in = torch.from_numpy(np.ascontiguousarray(grid)).cuda()
    d_out = torch.full_like(d_in, float("nan"))
    torch.cuda.synchronize()
    code = _lib.F64 if dtype == "f64" else _lib.F32
    _lib.check(lib.charming_jacobi2d_sweeps_noalloc(code, nx, ny, sweeps, d_in.data_ptr(),
                                                    d_out.data_ptr()),
               "charming_jacobi2d_sweeps_noalloc")
    return d_out.cpu().numpy()


def bits(a):
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_noalloc_matches_chare_entry_point_twice(rt, dtype):
    torch = pytest.importorskip("torch")
    npdt = np.float64 if dtype == "f64" else np.float32
    lib = rt.lib
    cases = [((301, 207), 37, 11), ((150, 90), 20, 12)]  # second call: smaller grid
    for (nx, ny), sweeps, seed in cases:
        g = seeded_grid(nx, ny, seed).astype(npdt)
        ref = chare_result(g, sweeps, dtype)
        out = noalloc_result(lib, torch, g, sweeps, dtype)
        assert np.array_equal(bits(out), bits(ref)), (nx, ny, sweeps)
        if dtype == "f64":  # and with the serial oracle itself
            assert np.array_equal(bits(out), bits(jacobi2d(g, sweeps))), (nx, ny, sweeps)


@pytest.mark.gpu
def test_noalloc_largest_grid_and_zero_sweeps(rt):
    torch = pytest.importorskip("torch")
    lib = rt.lib
    # (nx+2)*(ny+2)*8 == 16 MiB exactly: the largest FP64 grid accepted
    nx, ny = 2046, 1022
    g = seeded_grid(nx, ny, 5)
    out = noalloc_result(lib, torch, g, 3, "f64")
    assert np.array_equal(bits(out), bits(chare_result(g, 3, "f64")))
    out0 = noalloc_result(lib, torch, g, 0, "f64")
    assert np.array_equal(bits(out0), bits(g))


def test_noalloc_rejects_oversize_and_bad_arguments():
    """Checked before any CUDA call, so it runs without a GPU."""
    lib = _lib.load()
    fn = lib.charming_jacobi2d_sweeps_noalloc
    buf_a, buf_b = C.c_void_p(1 << 20), C.c_void_p(1 << 30)  # never dereferenced
    # one element past the 16 MiB scratch
    assert fn(_lib.F64, 2046, 1023, 1, buf_a, buf_b) == 14
    assert b"16 MiB" in lib.charming_last_error()
    assert fn(_lib.F32, 4094, 2046, 1, buf_a, buf_b) == 14
    assert fn(7, 10, 10, 1, buf_a, buf_b) == 14
    assert fn(_lib.F64, 0, 10, 1, buf_a, buf_b) == 14
    assert fn(_lib.F64, 10, 10, -1, buf_a, buf_b) == 14
    assert fn(_lib.F64, 10, 10, 1, None, buf_b) == 14
    assert fn(_lib.F64, 10, 10, 1, buf_a, C.c_void_p((1 << 20) + 64)) == 14  # overlap
    # element pointers not aligned to the element size
    assert fn(_lib.F64, 10, 10, 1, C.c_void_p((1 << 20) + 4), buf_b) == 14
    assert b"aligned" in lib.charming_last_error()
    assert fn(_lib.F32, 10, 10, 1, buf_a, C.c_void_p((1 << 30) + 2)) == 14
    # sizes whose +2 would overflow a 32-bit int
    assert fn(_lib.F64, 2**31 - 1, 1, 1, buf_a, buf_b) == 14
    assert fn(_lib.F32, 1, 2**31 - 2, 1, buf_a, buf_b) == 14
    assert b"16 MiB" in lib.charming_last_error()
