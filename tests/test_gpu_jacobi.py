"""GPU parity tests of the Jacobi chares against the CPU oracle (bit-exact)."""
import ctypes as C

import numpy as np
import pytest

from charming_b200.jacobi import Jacobi2D, Problem, initial_grid
from oracle import jacobi as oj
from oracle.jacobi import seeded_grid


def jac64(grid, sweeps):
    return oj.jacobi2d(np.asarray(grid, dtype=np.float64), sweeps)


def oracle_lib():
    return oj.lib()

pytestmark = pytest.mark.gpu


def jac32(grid, sweeps):
    g = np.ascontiguousarray(grid, dtype=np.float32).copy()
    ny, nx = g.shape[0] - 2, g.shape[1] - 2
    oracle_lib().oracle_jacobi2d_f32(g.ctypes.data_as(C.POINTER(C.c_float)), nx, ny, sweeps, 0)
    return g


def bits(a):
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


@pytest.mark.parametrize("pipeline", [True, False])
def test_c1_512_fp64_bit_exact(rt, pipeline):
    """C1: 512^2 interior, top 1 / others 0, 4x4 chares of 128^2, 100 sweeps,
    one halo exchange per sweep as in the reference."""
    p = Problem(512, 512, 100, px=4, py=4, bc=(1.0, 0.0, 0.0, 0.0))
    with Jacobi2D([p], pipeline=pipeline, depth=1) as j:
        j.run()
        out = j.store(0)
        assert j.result(0).sweeps == 100
        info = j.info()
        assert info["n_chares"] == 16 and info["halo_msgs_per_sweep"] == 48
    ref = jac64(initial_grid(512, 512, p.bc), 100)
    assert np.array_equal(bits(out), bits(ref))
    st = rt.last_stats()
    assert st.status == 0
    assert st.delivered >= 100 * 48


@pytest.mark.parametrize("nx,ny,px,py,sweeps,tile_w", [
    (333, 201, 5, 3, 17, 0),      # uneven splits
    (1000, 77, 7, 2, 9, 0),
    (64, 64, 1, 1, 25, 0),        # single chare, no halos
    (50, 700, 1, 9, 11, 0),       # tall
    (333, 97, 2, 2, 13, 64),      # several column tiles per chare
    (2500, 40, 2, 1, 5, 0),       # chare wider than one tile
    (1, 1, 1, 1, 3, 0),           # smallest grid
    (7, 300, 7, 3, 6, 0),         # one-column chares
])
@pytest.mark.parametrize("pipeline", [True, False])
def test_seeded_grids_fp64_bit_exact(rt, nx, ny, px, py, sweeps, tile_w, pipeline):
    g = seeded_grid(nx, ny, nx * 31 + ny)
    p = Problem(nx, ny, sweeps, px=px, py=py)
    with Jacobi2D([p], pipeline=pipeline, tile_w=tile_w) as j:
        j.load(0, g)
        j.run()
        out = j.store(0)
    assert np.array_equal(bits(out), bits(jac64(g, sweeps)))


def test_batched_uneven_problems_one_launch(rt):
    rng = np.random.default_rng(5)
    probs, grids = [], []
    for k in range(12):
        nx, ny = (int(x) for x in rng.integers(20, 300, size=2))
        probs.append(Problem(nx, ny, int(rng.integers(1, 40)), bc=tuple(rng.random(4))))
    with Jacobi2D(probs, chare_side=64) as j:
        j.run()
        for k, p in enumerate(probs):
            out = j.store(k)
            ref = jac64(initial_grid(p.nx, p.ny, p.bc), p.max_sweeps)
            assert np.array_equal(bits(out), bits(ref)), k
            assert j.result(k).sweeps == p.max_sweeps


@pytest.mark.parametrize("pipeline", [True, False])
def test_fp32_bit_exact(rt, pipeline):
    g = seeded_grid(300, 180, 77).astype(np.float32)
    p = Problem(300, 180, 40, px=3, py=2)
    with Jacobi2D([p], dtype="f32", pipeline=pipeline) as j:
        j.load(0, g)
        j.run()
        out = j.store(0)
    assert np.array_equal(bits(out), bits(jac32(g, 40)))


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_residual_stop_rule(rt, dtype):
    """Stops at a multiple of check_every once ||r|| <= tol * ||r_0||; the grid
    equals the oracle after that many sweeps; norms match the oracle."""
    lib = oracle_lib()
    nx, ny, K = 96, 80, 10
    p = Problem(nx, ny, 3000, px=3, py=2, check_every=K, tol=0.05, bc=(1.0, 0.25, 0.5, 0.0))
    npdt = np.float64 if dtype == "f64" else np.float32
    with Jacobi2D([p], dtype=dtype) as j:
        j.run()
        out = j.store(0)
        r = j.result(0)
    assert 0 < r.sweeps < 3000 and r.sweeps % K == 0
    g0 = initial_grid(nx, ny, p.bc, npdt)
    ref = jac64(g0, r.sweeps) if dtype == "f64" else jac32(g0, r.sweeps)
    assert np.array_equal(bits(out), bits(ref))
    res2 = (lib.oracle_residual2_f64 if dtype == "f64" else lib.oracle_residual2_f32)
    ptr_t = C.POINTER(C.c_double if dtype == "f64" else C.c_float)
    r0 = np.sqrt(res2(np.ascontiguousarray(g0).ctypes.data_as(ptr_t), nx, ny))
    assert r.res0 == pytest.approx(r0, rel=1e-12)
    # the decision taken at check c = sweeps/K - 1 said stop
    g_chk = jac64(g0, r.sweeps - K) if dtype == "f64" else jac32(g0, r.sweeps - K)
    rc = np.sqrt(res2(np.ascontiguousarray(g_chk).ctypes.data_as(ptr_t), nx, ny))
    assert r.res_last == pytest.approx(rc, rel=1e-12)
    assert rc <= 0.05 * r0
    g_prev = jac64(g0, r.sweeps - 2 * K) if dtype == "f64" else jac32(g0, r.sweeps - 2 * K)
    rp = np.sqrt(res2(np.ascontiguousarray(g_prev).ctypes.data_as(ptr_t), nx, ny))
    assert rp > 0.05 * r0


def test_graph_replay_matches(rt):
    p = Problem(256, 256, 30, px=2, py=2, bc=(1.0, 0.0, 0.5, 0.0))
    ref = jac64(initial_grid(256, 256, p.bc), 30)
    with Jacobi2D([p], use_graph=True) as j:
        for _ in range(3):
            j.init()
            j.run()
            assert np.array_equal(bits(j.store(0)), bits(ref))


def test_jacobi1d_bit_exact(rt):
    n, w, sweeps = 9, 37, 50
    out, _ = rt.jacobi1d(n, w, sweeps)
    a = np.zeros(n * w + 4)
    a[:2] = 10.0
    a[-2:] = 10.0
    lib = oracle_lib()
    lib.oracle_jacobi1d_f64(a.ctypes.data_as(C.POINTER(C.c_double)), n * w, sweeps)
    assert np.array_equal(out.view(np.uint64), a.view(np.uint64))


@pytest.mark.parametrize("pipeline", [True, False])
def test_halo_refnum_mode_bit_exact(rt, pipeline):
    """halo_mode 1: halos tagged refnum = sweep, early ones parked in the stash."""
    g = seeded_grid(200, 150, 12)
    p = Problem(200, 150, 21, px=4, py=3)
    with Jacobi2D([p], pipeline=pipeline, halo_mode=1) as j:
        j.load(0, g)
        j.run()
        out = j.store(0)
    assert np.array_equal(bits(out), bits(jac64(g, 21)))


def test_many_chares_per_pe(rt):
    """Over-decomposition: several chares per PE, uneven placement."""
    g = seeded_grid(700, 610, 99)
    p = Problem(700, 610, 15, px=23, py=19)
    with Jacobi2D([p], balance=False) as j:
        j.load(0, g)
        j.run()
        out = j.store(0)
        assert j.info()["max_chares_per_pe"] >= 2
    assert np.array_equal(bits(out), bits(jac64(g, 15)))


@pytest.mark.parametrize("corner_msgs", [False, True])
@pytest.mark.parametrize("depth", [2, 3, 4, 5, 6, 8])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_multi_sweep_passes_bit_exact(rt, depth, dtype, corner_msgs, monkeypatch):
    """depth sweeps per halo exchange (ghost zones of that depth): the same
    bits as one sweep per exchange. The corners travel in the second phase
    of a two-phase exchange (left/right halos, then top/bottom halos that
    carry the ghost columns), or, with CHARMING_HALO_CORNERS=1, in messages
    from the diagonal neighbours. Sweep counts that are not multiples of the
    depth end with a shorter pass."""
    monkeypatch.setenv("CHARMING_HALO_CORNERS", "1" if corner_msgs else "0")
    npdt = np.float64 if dtype == "f64" else np.float32
    for (nx, ny, px, py, sweeps) in [(333, 201, 5, 3, 37), (1000, 77, 7, 2, 9), (50, 700, 1, 9, 11),
                                     (2500, 40, 2, 1, 6), (300, 180, 3, 2, 40)]:
        g = seeded_grid(nx, ny, nx * 7 + ny + depth).astype(npdt)
        with Jacobi2D([Problem(nx, ny, sweeps, px=px, py=py)], dtype=dtype, depth=depth) as j:
            j.load(0, g)
            j.run()
            out = j.store(0)
            info = j.info()
        ref = jac64(g, sweeps) if dtype == "f64" else jac32(g, sweeps)
        assert np.array_equal(bits(out), bits(ref)), (nx, ny, px, py, sweeps)
        corners = 4 * (px - 1) * (py - 1) if corner_msgs else 0
        edges = 2 * (px - 1) * py + 2 * px * (py - 1)
        assert info["halo_msgs_per_sweep"] == edges + corners


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_multi_sweep_residual_stop_rule(rt, dtype):
    """Residual checks every 10 sweeps with passes of 4: passes 4, 4, 2 so
    every check starts a pass; stops where one-sweep exchanges stop."""
    nx, ny, K = 96, 80, 10
    p = Problem(nx, ny, 3000, px=3, py=2, check_every=K, tol=0.05, bc=(1.0, 0.25, 0.5, 0.0))
    npdt = np.float64 if dtype == "f64" else np.float32
    with Jacobi2D([p], dtype=dtype, depth=4) as j:
        j.run()
        out = j.store(0)
        r = j.result(0)
    with Jacobi2D([p], dtype=dtype, depth=1) as j:
        j.run()
        r1 = j.result(0)
    assert r.sweeps == r1.sweeps and r.sweeps % K == 0
    g0 = initial_grid(nx, ny, p.bc, npdt)
    ref = jac64(g0, r.sweeps) if dtype == "f64" else jac32(g0, r.sweeps)
    assert np.array_equal(bits(out), bits(ref))
    assert r.res0 == pytest.approx(r1.res0, rel=1e-12)


def test_autotune_reinit_and_configs(rt):
    """The autotuner re-initialises the runtime per candidate (chare side,
    PEs per SM, ring depth); every candidate gives the same grid bit for
    bit, and the default runtime comes back afterwards."""
    from charming_b200.batch import Candidate, autotune, uneven_set
    from charming_b200.runtime import Runtime
    probs = uneven_set(seed=7, n=6, lo=32, hi=300, max_sweeps=30)
    ref = [jac64(initial_grid(p.nx, p.ny, p.bc), 30) for p in probs]
    cands = [Candidate(64, 1, 1 << 20), Candidate(128, 2, 4 << 20), Candidate(256, 1, 4 << 20)]
    grids = []
    for c in cands:
        Runtime(**c.runtime_config())
        with Jacobi2D(probs, chare_side=c.chare_side, use_graph=True) as j:
            j.run()
            grids.append([j.store(i) for i in range(len(probs))])
    for g in grids:
        for a, b in zip(ref, g):
            assert np.array_equal(bits(a), bits(b))
    tune = autotune(probs, "f64", candidates=cands)
    assert tune.best.glups > 0 and all(c.glups > 0 for c in tune.tried)
    Runtime()  # default configuration for the tests that follow
    assert Runtime._active.info["n_pes"] == rt.info["n_pes"]


def test_headline_configuration_bit_exact(rt):
    """The benchmark's headline problem exactly as bench.py runs it: 8192^2
    FP64, top 1 / others 0, the decomposition bench.py picks (4 x 37 chares
    on a B200), 6 sweeps per halo exchange, balanced row runs, 100 sweeps,
    compared bit for bit with the OpenMP oracle (bit-identical to the serial
    one) on all host cores."""
    import os

    import bench
    px, py = bench.choose_decomposition(rt.n_pes, 8192, 8192)
    p = Problem(8192, 8192, 100, px=px, py=py, bc=(1.0, 0.0, 0.0, 0.0))
    with Jacobi2D([p], dtype="f64", pipeline=False, balance=True, tile_w=0, depth=0) as j:
        j.run()
        out = j.store(0)
        assert j.result(0).sweeps == 100
    ref = oj.jacobi2d(initial_grid(8192, 8192, p.bc), 100, threads=os.cpu_count() or 1)
    assert np.array_equal(bits(out), bits(ref))



@pytest.mark.parametrize("use_graph", [False, True])
def test_solve_stream_matches_load_run_store(rt, use_graph):
    """Pipelined solves (input copy of the next and result copy of the
    previous solve overlapping each solve) give each grid's own result."""
    p = Problem(300, 220, 23, px=3, py=2)
    grids = [seeded_grid(300, 220, s) for s in (1, 2, 3, 4, 5)]
    outs = [np.empty_like(g) for g in grids]
    with Jacobi2D([p], use_graph=use_graph) as j:
        ms = j.solve_stream(0, grids, outs)
        assert ms > 0
        for g, o in zip(grids, outs):
            assert np.array_equal(bits(o), bits(jac64(g, 23)))
