"""CPU check of the Jacobi chare code: jacobi2d.cu compiled for the host
(tests/emu) and run on an in-process stand-in for the runtime. Two builds:
one host thread per PE under AddressSanitizer/UBSan (many PEs, random
message orders), and one PE block of many host threads under
ThreadSanitizer, with call-site-checked barriers, lockstep warps and a model
of mbarriers and asynchronous bulk copies for the TMA sweep. The grid must
match the serial oracle bit for bit and the residual stop rule must stop
where the oracle says."""
import os
import subprocess

import numpy as np
import pytest

from charming_b200.jacobi import initial_grid
from oracle import jacobi as oj
from oracle.jacobi_protocol import ProtocolError, Sim

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "build", "emu", "jacobi_emu")
EMU_MT = os.path.join(ROOT, "build", "emu", "jacobi_emu_mt")


@pytest.fixture(scope="module")
def emu():
    r = subprocess.run(["make", "-s"], cwd=os.path.join(ROOT, "tests", "emu"), capture_output=True,
                       text=True)
    if r.returncode != 0:
        pytest.fail(r.stdout[-3000:] + r.stderr[-3000:])
    return EMU


def run_emu(emu, nx, ny, px, py, max_sweeps, K, tol, dtype, n_pes, halo, bc, seed=1,
            threads=1, pipeline=0, tile_w=0, depth=1, balance=0):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0", TSAN_OPTIONS="halt_on_error=1")
    args = [emu] + [str(x) for x in (nx, ny, px, py, max_sweeps, K, tol, dtype, n_pes, halo)]
    args += [str(b) for b in bc] + [str(seed), str(threads), str(pipeline), str(tile_w),
                                    str(depth), str(balance)]
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
    # nx, ny, px, py, max_sweeps, K, tol, dtype, n_pes, halo_mode, depth, balance
    (96, 80, 3, 2, 3000, 10, 0.05, 0, 6, 0, 1, 0),
    (96, 80, 3, 2, 3000, 10, 0.05, 1, 2, 1, 1, 1),
    (200, 150, 4, 3, 400, 1, 0.2, 0, 5, 0, 1, 0),
    (333, 201, 5, 3, 300, 7, 0.01, 0, 8, 0, 1, 1),
    (64, 64, 1, 1, 100, 10, 0.1, 0, 1, 0, 1, 0),
    (50, 700, 1, 9, 500, 3, 0.3, 1, 4, 1, 1, 0),
    (120, 120, 6, 6, 60, 0, 0.0, 0, 7, 0, 1, 0),
    (31, 17, 4, 2, 60, 2, 0.5, 0, 3, 1, 1, 0),
    # several sweeps per exchange: deep ghost zones, corner halos
    (96, 80, 3, 2, 3000, 10, 0.05, 0, 6, 0, 4, 1),
    (333, 201, 5, 3, 300, 7, 0.01, 1, 8, 1, 3, 0),
    (200, 150, 4, 3, 41, 0, 0.0, 0, 5, 0, 2, 1),
    (50, 700, 1, 9, 500, 3, 0.3, 1, 4, 1, 4, 0),
    (31, 17, 4, 2, 60, 2, 0.5, 0, 3, 0, 4, 0),
    (120, 120, 6, 6, 61, 0, 0.0, 1, 7, 1, 4, 1),
    (96, 80, 3, 2, 3000, 10, 0.05, 1, 6, 0, 5, 1),   # depth 5: passes 5 + 5 per check
    (200, 150, 4, 3, 43, 0, 0.0, 0, 5, 1, 5, 0),
    (96, 80, 3, 2, 3000, 10, 0.05, 0, 6, 0, 0, 0),   # automatic depth for a period of 10
])
def test_chare_code_on_cpu(emu, cfg):
    nx, ny, px, py, ms, K, tol, dt, npes, halo, depth, bal = cfg
    bc = (0.3, 0.9, 0.1, 0.7)
    rc, f, err = run_emu(emu, nx, ny, px, py, ms, K, tol, dt, npes, halo, bc, depth=depth,
                         balance=bal)
    assert rc == 0 and f.get("status") == "0" and f.get("exact") == "1", (f, err[-2000:])
    assert int(f["done"]) == px * py
    if K > 0:
        assert int(f["sweeps"]) == expected_stop(nx, ny, K, tol, ms, bc, dt)


@pytest.mark.parametrize("two_phase", [False, True])
@pytest.mark.parametrize("px,py,K,mx,stop_at", [
    (3, 2, 10, 3000, 5), (4, 4, 1, 50, 7), (5, 3, 3, 40, 100), (1, 6, 10, 55, 2), (7, 1, 0, 30, 0),
])
def test_protocol_model_random_orders(px, py, K, mx, stop_at, two_phase):
    ends = set()
    for seed in range(25):
        ends.add(Sim(px, py, K, mx, stop_at, seed, two_phase=two_phase).run())
    assert len(ends) == 1


@pytest.mark.parametrize("cfg", [
    # nx, ny, px, py, max_sweeps, K, tol, dtype, halo_mode, threads, pipeline, tile_w, depth
    (48, 40, 3, 2, 300, 5, 0.2, 0, 0, 64, 1, 0, 1),     # the residual stop rule, TMA sweep
    (48, 40, 3, 2, 300, 5, 0.2, 1, 1, 32, 0, 0, 1),
    (120, 90, 4, 3, 12, 1, 0.2, 0, 0, 64, 1, 64, 1),    # several column tiles
    (333, 97, 2, 2, 13, 0, 0.0, 0, 1, 96, 1, 0, 1),
    (50, 70, 1, 3, 40, 3, 0.3, 1, 0, 32, 1, 0, 1),
    (64, 64, 1, 1, 25, 5, 0.1, 0, 0, 40, 0, 0, 1),      # single chare, odd block size
    (48, 40, 3, 2, 300, 5, 0.2, 0, 0, 64, 0, 0, 4),     # multi-sweep passes (warp wavefront)
    (150, 90, 3, 3, 13, 4, 0.01, 1, 1, 64, 0, 0, 3),
    (300, 100, 1, 1, 17, 0, 0.0, 0, 0, 96, 0, 0, 2),
    (1100, 40, 2, 1, 9, 0, 0.0, 1, 0, 128, 0, 0, 4),
    (48, 40, 3, 2, 300, 10, 0.2, 1, 0, 64, 0, 0, 5),
    (200, 60, 2, 2, 31, 0, 0.0, 0, 0, 64, 0, 0, 6),     # deeper passes: strips and row
    (150, 50, 1, 2, 27, 0, 0.0, 1, 1, 96, 0, 0, 7),     # runs overlap by more vectors
    (260, 44, 2, 1, 40, 10, 0.01, 0, 0, 64, 0, 0, 8),
])
def test_chare_code_threaded_block(emu, cfg):
    """One PE block of many threads: barriers reached from different call
    sites, races between thread 0 and the rest, and misuse of mbarriers or
    bulk copies abort the run."""
    nx, ny, px, py, ms, K, tol, dt, halo, thr, pl, tw, depth = cfg
    bc = (1.0, 0.25, 0.5, 0.0)
    rc, f, err = run_emu(EMU_MT, nx, ny, px, py, ms, K, tol, dt, 1, halo, bc,
                         threads=thr, pipeline=pl, tile_w=tw, depth=depth)
    assert "ThreadSanitizer" not in err and "divergence" not in err, err[-3000:]
    assert rc == 0 and f.get("status") == "0" and f.get("exact") == "1", (f, err[-2000:])
    assert int(f["done"]) == px * py
    if K > 0:
        assert int(f["sweeps"]) == expected_stop(nx, ny, K, tol, ms, bc, dt)
