"""GPU tests of the solve server (charming_serve_*): every result equals
the serial oracle bit for bit (FP64 sweeps, and FP32 sweeps with the FP64
residual and stop rule), each request gives the same result alone and in a
mix of concurrent requests, the batched path gives the same result for the
same problem, and admission keeps to the HBM budget, the request slots and
the worker pool."""
import ctypes as C

import numpy as np
import pytest

from charming_b200.jacobi import Jacobi2D, Problem, initial_grid
from charming_b200.serve import Server
from oracle import jacobi as oj

pytestmark = pytest.mark.gpu


def jac64(grid, sweeps):
    return oj.jacobi2d(np.asarray(grid, dtype=np.float64), sweeps)


def jac32(grid, sweeps):
    g = np.ascontiguousarray(grid, dtype=np.float32).copy()
    ny, nx = g.shape[0] - 2, g.shape[1] - 2
    oj.lib().oracle_jacobi2d_f32(g.ctypes.data_as(C.POINTER(C.c_float)), nx, ny, sweeps, 0)
    return g


def bits(a):
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def mixed(seed, n, lo, hi, max_sweeps, check_every=0, tol=0.0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx, ny = (int(x) for x in np.exp(rng.uniform(np.log(lo), np.log(hi), 2)).round())
        out.append(Problem(nx, ny, max_sweeps, check_every=check_every, tol=tol,
                           bc=tuple(float(v) for v in rng.uniform(0, 1, 4))))
    return out


def serve_all(server, probs, tag0=0):
    for i, p in enumerate(probs):
        server.submit(p, tag0 + i)
    done = server.wait(range(tag0, tag0 + len(probs)))
    grids = []
    for i in range(len(probs)):
        grids.append(server.fetch(tag0 + i).copy())
        server.release(tag0 + i)
    return [done[tag0 + i] for i in range(len(probs))], grids


def test_serve_fp64_matches_oracle(rt):
    probs = mixed(3, 10, 20, 300, 60)
    with Server(1 << 30, max_inflight=8, workers_per_pe=4, chare_side=64, dtype="f64",
                deadline_s=60) as s:
        comps, grids = serve_all(s, probs)
        stats = s.stop()
    for p, c, g in zip(probs, comps, grids):
        assert c.status == 0 and c.sweeps == 60
        ref = jac64(initial_grid(p.nx, p.ny, p.bc), 60)
        assert np.array_equal(bits(g), bits(ref)), (p.nx, p.ny)
    assert stats["completed"] == len(probs) and stats["peak_inflight"] <= 8
    assert rt.last_stats().status == 0


def test_serve_alone_equals_mix_fp32(rt):
    """FP32 sweeps with the FP64 residual every 10 sweeps; some requests stop
    early on tol. Alone, in a mix, and through the batched path: the same
    sweeps, residuals and grids, equal to the FP32 oracle run for the same
    sweep count."""
    probs = mixed(5, 12, 40, 500, 300, check_every=10, tol=0.05)
    for p in probs[::2]:
        p.tol = 1e-4  # runs to the cap
    with Server(1 << 30, max_inflight=16, workers_per_pe=8, chare_side=64, dtype="f32",
                deadline_s=60) as s:
        alone = [serve_all(s, [p], tag0=100 + i) for i, p in enumerate(probs)]
        mix_c, mix_g = serve_all(s, probs, tag0=1000)
        stats = s.stop()
    assert stats["peak_inflight"] > 1  # the mix ran concurrently
    with Jacobi2D(probs, dtype="f32", chare_side=64) as j:
        j.run()
        batch = [(j.result(i), j.store(i)) for i in range(len(probs))]
    early = 0
    for i, p in enumerate(probs):
        (ca,), (ga,) = alone[i]
        cm, gm = mix_c[i], mix_g[i]
        rb, gb = batch[i]
        assert ca.sweeps == cm.sweeps == rb.sweeps
        assert ca.res_last == cm.res_last == rb.res_last and ca.res0 == cm.res0 == rb.res0
        assert np.array_equal(bits(ga), bits(gm)) and np.array_equal(bits(ga), bits(gb))
        ref = jac32(initial_grid(p.nx, p.ny, p.bc, dtype=np.float32), ca.sweeps)
        assert np.array_equal(bits(ga), bits(ref)), (i, p.nx, p.ny, ca.sweeps)
        early += ca.sweeps < p.max_sweeps
    assert 0 < early < len(probs)  # the stop rule fired for some, not all


def test_serve_admission_under_budget(rt):
    """A budget that holds only a few grids at once: requests queue, are
    admitted as memory is released, and all complete."""
    probs = [Problem(256, 256, 40, bc=(1.0, 0.0, 0.5, 0.25)) for _ in range(10)]
    budget = 3 * 2 * 270 * 300 * 8 + (1 << 16)  # about three 256^2 FP64 requests
    with Server(budget, max_inflight=8, workers_per_pe=8, chare_side=128, dtype="f64",
                deadline_s=60) as s:
        for i, p in enumerate(probs):
            s.submit(p, i)
        got = {}
        import time
        t_end = time.monotonic() + 60
        while len(got) < len(probs):
            for c in s.poll():
                got[c.tag] = c
                g = s.fetch(c.tag)
                s.release(c.tag)
                assert np.array_equal(bits(g), bits(jac64(initial_grid(256, 256, probs[0].bc), 40)))
            assert time.monotonic() < t_end
        stats = s.stop()
    assert stats["peak_bytes"] <= budget
    assert 1 <= stats["peak_inflight"] < len(probs)
    assert all(got[i].admit_s >= got[i].submit_s for i in got)
    # queued requests waited for memory: some were admitted well after submission
    assert max(got[i].admit_s - got[i].submit_s for i in got) > 0
