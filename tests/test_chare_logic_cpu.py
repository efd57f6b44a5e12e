"""CPU check of the Jacobi chare code: jacobi2d.cu compiled for the host
(tests/emu) and run on an in-process stand-in for the runtime, one host
thread per PE, under AddressSanitizer/UBSan; the grid must match the serial
oracle bit for bit and the residual stop rule must stop where the oracle
says."""
import os
import subprocess

import numpy as np
import pytest

from charming_b200.jacobi import initial_grid
from oracle import jacobi as oj
from oracle.jacobi_protocol import ProtocolError, Sim

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "build", "emu", "jacobi_emu")


@pytest.fixture(scope="module")
def emu():
    r = subprocess.run(["make", "-s"], cwd=os.path.join(ROOT, "tests", "emu"), capture_output=True,
                       text=True)
    if r.returncode != 0:
        pytest.fail(r.stdout[-3000:] + r.stderr[-3000:])
    return EMU


def run_emu(emu, nx, ny, px, py, max_sweeps, K, tol, dtype, n_pes, halo, bc, seed=1):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0")
    args = [emu] + [str(x) for x in (nx, ny, px, py, max_sweeps, K, tol, dtype, n_pes, halo)]
    args += [str(b) for b in bc] + [str(seed)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300, env=env)
    line = r.stdout.strip().splitlines()[-1] if r.stdout.strip() else ""
    fields = dict(kv.split("=", 1) for kv in line.split())
    return r.returncode, fields, r.stderr


def expected_stop(nx, ny, K, tol, max_sweeps, bc, dtype):
    """Sweep at which the stop rule fires: the decision of check c (residual
    of u_{cK}) is applied at sweep (c+1)K."""
    g = initial_grid(nx, ny, bc, np.float64 if dtype == 0 else np.float32)
    r0 = oj.residual(g)
    u = g
    for c in range(max_sweeps // K + 1):
        if c:
            u = oj.jacobi2d(u, K)
        if (c + 1) * K > max_sweeps:
            return max_sweeps
        if tol > 0 and oj.residual(u) <= tol * r0:
            return (c + 1) * K
    return max_sweeps


@pytest.mark.parametrize("cfg", [
    # nx, ny, px, py, max_sweeps, K, tol, dtype, n_pes, halo_mode
    (96, 80, 3, 2, 3000, 10, 0.05, 0, 6, 0),
    (96, 80, 3, 2, 3000, 10, 0.05, 1, 2, 1),
    (200, 150, 4, 3, 400, 1, 0.2, 0, 5, 0),
    (333, 201, 5, 3, 300, 7, 0.01, 0, 8, 0),
    (64, 64, 1, 1, 100, 10, 0.1, 0, 1, 0),
    (50, 700, 1, 9, 500, 3, 0.3, 1, 4, 1),
    (120, 120, 6, 6, 60, 0, 0.0, 0, 7, 0),
    (31, 17, 4, 2, 60, 2, 0.5, 0, 3, 1),
])
def test_chare_code_on_cpu(emu, cfg):
    nx, ny, px, py, ms, K, tol, dt, npes, halo = cfg
    bc = (0.3, 0.9, 0.1, 0.7)
    rc, f, err = run_emu(emu, nx, ny, px, py, ms, K, tol, dt, npes, halo, bc)
    assert rc == 0 and f.get("status") == "0" and f.get("exact") == "1", (f, err[-2000:])
    assert int(f["done"]) == px * py
    if K > 0:
        assert int(f["sweeps"]) == expected_stop(nx, ny, K, tol, ms, bc, dt)


@pytest.mark.parametrize("px,py,K,mx,stop_at", [
    (3, 2, 10, 3000, 5), (4, 4, 1, 50, 7), (5, 3, 3, 40, 100), (1, 6, 10, 55, 2), (7, 1, 0, 30, 0),
])
def test_protocol_model_random_orders(px, py, K, mx, stop_at):
    ends = set()
    for seed in range(25):
        ends.add(Sim(px, py, K, mx, stop_at, seed).run())
    assert len(ends) == 1
