"""CPU tests: the oracle against known answers and golden fixtures."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import msgmodel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def oracle_lib():
    path = os.path.join(ROOT, "oracle", "liboracle_jacobi.so")
    if not os.path.exists(path):
        import subprocess
        subprocess.run(["make"], cwd=os.path.join(ROOT, "oracle"), check=True, capture_output=True)
    lib = C.CDLL(path)
    dp, fp, i = C.POINTER(C.c_double), C.POINTER(C.c_float), C.c_int
    lib.oracle_jacobi2d_f64.argtypes = [dp, i, i, i]
    lib.oracle_jacobi2d_f64_omp.argtypes = [dp, i, i, i, i]
    lib.oracle_jacobi2d_f32.argtypes = [fp, i, i, i, i]
    lib.oracle_residual2_f64.argtypes = [dp, i, i]
    lib.oracle_residual2_f64.restype = C.c_double
    lib.oracle_residual2_f32.argtypes = [fp, i, i]
    lib.oracle_residual2_f32.restype = C.c_double
    lib.oracle_jacobi1d_f64.argtypes = [dp, i, i]
    return lib


def jac64(grid, sweeps, threads=0):
    g = np.ascontiguousarray(grid, dtype=np.float64).copy()
    lib = oracle_lib()
    ny, nx = g.shape[0] - 2, g.shape[1] - 2
    ptr = g.ctypes.data_as(C.POINTER(C.c_double))
    if threads:
        lib.oracle_jacobi2d_f64_omp(ptr, nx, ny, sweeps, threads)
    else:
        lib.oracle_jacobi2d_f64(ptr, nx, ny, sweeps)
    return g


def seeded_grid(nx, ny, seed):
    k = np.arange((nx + 2) * (ny + 2), dtype=np.uint64)
    with np.errstate(over="ignore"):
        v = msgmodel.mix64((np.uint64(seed) << np.uint64(32)) + k) >> np.uint64(11)
    return (v.astype(np.float64) * (1.0 / 9007199254740992.0)).reshape(ny + 2, nx + 2)


# ---- generators -------------------------------------------------------------
def test_splitmix64_published_sequence():
    # Reference outputs of SplitMix64 (Vigna) for seed 0.
    seq = msgmodel.splitmix64_sequence(0, 2)
    assert seq == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4]


def test_checksum_position_dependent_and_length():
    a = bytes(range(64))
    b = a[8:16] + a[:8] + a[16:]
    assert msgmodel.checksum(a) != msgmodel.checksum(b)
    assert msgmodel.checksum(a[:13]) != msgmodel.checksum(a[:13] + b"\0")
    assert msgmodel.checksum(b"") == 0


def test_fanout_checksums_vectorised_match_scalar():
    n, msgs, payload, seed = 7, 5, 64, 123
    for mode in (0, 1):
        vec = msgmodel.fanout_checksums(n, msgs, payload, seed, mode)
        for s in range(n):
            for k in range(msgs):
                p = msgmodel.fanout_payload(seed, n, msgs, payload, s, k, mode)
                assert int(vec[s, k]) == msgmodel.checksum(p)


def test_fanout_expected_counts_sum():
    c = msgmodel.fanout_expected_counts(4096, 16, 99)
    assert c.sum() == 4096 * 16
    assert np.all(c.sum(axis=0) == 4096)


def test_fanout_checker_accepts_model_log_and_rejects_faults():
    n, msgs, payload, seed, mode = 50, 6, 32, 5, 1
    dst = msgmodel.fanout_destinations(n, msgs, seed)
    cs = msgmodel.fanout_checksums(n, msgs, payload, seed, mode)
    recs, seqs = [], {}
    # senders interleaved round-robin over k: a valid FIFO / refnum-ordered log
    for k in range(msgs):
        for s in range(n):
            d = int(dst[s, k])
            q = seqs.get(d, 0)
            seqs[d] = q + 1
            c = int(cs[s, k])
            recs.append([d, s, k, k, q, c & 0xFFFFFFFF, c >> 32, k])
    log = np.array(recs, dtype=np.uint32)
    assert msgmodel.check_fanout_log(log, n, msgs, payload, seed, mode).ok
    bad = log.copy()
    bad[3, 5] ^= 1  # corrupt one checksum (planted fault, CPU only)
    assert not msgmodel.check_fanout_log(bad, n, msgs, payload, seed, mode).ok
    dropped = log[1:]
    assert not msgmodel.check_fanout_log(dropped, n, msgs, payload, seed, mode).ok
    # swap two deliveries of the same pair -> FIFO violation
    pairs = {}
    for i, r in enumerate(log):
        pairs.setdefault((r[0], r[1]), []).append(i)
    i, j = next(v for v in pairs.values() if len(v) >= 2)[:2]
    sw = log.copy()
    sw[[i, j], 4] = sw[[j, i], 4]
    assert not msgmodel.check_fanout_log(sw, n, msgs, payload, seed, mode).ok


# ---- messaging known answers (reference example behaviour) -----------------
def test_refnum_model_known_answer():
    assert msgmodel.refnum_scenario(False) == [1, 0]
    assert msgmodel.refnum_scenario(True) == [1, 0]


def test_hello_model_known_answer():
    assert msgmodel.hello_chain(3) == [0, 1, 2, 3, 4, 5]


def test_receiver_model_fifo_within_refnum():
    seen = []

    def em(model, m):
        seen.append(m.payload)
        if m.payload == "b0":
            model.set_refnum(0, 1)

    rm = msgmodel.ReceiverModel({0: 0}, em)
    for m in [msgmodel.Msg(0, 1, "a1"), msgmodel.Msg(0, 1, "a2"), msgmodel.Msg(0, 0, "b0"),
              msgmodel.Msg(0, 1, "a3")]:
        rm.arrive(m)
    assert seen == ["b0", "a1", "a2", "a3"]


# ---- Jacobi oracle -----------------------------------------------------------
def test_jacobi_hand_known_answer():
    g = np.zeros((5, 5))
    g[0, :] = 1.0  # top boundary
    out = jac64(g, 1)
    exp = np.zeros((5, 5))
    exp[0, :] = 1.0
    exp[1, 1:4] = 0.2
    assert np.array_equal(out, exp)
    out2 = jac64(g, 2)
    # second sweep, row 1: (c + l + r + u + d) * 0.2 in that order
    c = 0.2
    assert out2[1, 2] == (c + c + c + 1.0 + 0.0) * 0.2
    assert out2[1, 1] == (c + 0.0 + c + 1.0 + 0.0) * 0.2
    assert out2[2, 2] == (0.0 + 0.0 + 0.0 + c + 0.0) * 0.2


def test_jacobi_openmp_bit_identical_to_serial():
    g = seeded_grid(97, 61, 3)
    assert np.array_equal(jac64(g, 25), jac64(g, 25, threads=4))


def test_jacobi_boundary_ring_fixed():
    g = seeded_grid(33, 17, 9)
    out = jac64(g, 10)
    assert np.array_equal(out[0], g[0]) and np.array_equal(out[-1], g[-1])
    assert np.array_equal(out[:, 0], g[:, 0]) and np.array_equal(out[:, -1], g[:, -1])


def _round_f32(q) -> np.float32:
    """The float32 nearest the exact rational q (ties to even)."""
    from fractions import Fraction
    c = np.float32(float(q))
    best = None
    for v in (np.nextafter(c, np.float32(-np.inf)), c, np.nextafter(c, np.float32(np.inf))):
        d = abs(Fraction(float(v)) - q)
        if best is None or d < best[0] or (d == best[0] and int(v.view(np.uint32)) % 2 == 0):
            best = (d, v)
    return best[1]


def test_jacobi_f32_fma_split_of_the_factor():
    """FP32 sweeps: float sum s (left to right), then fma(s, C_HI, s * C_LO)
    with C_HI = 0.2f and C_LO the float nearest 0.2 - C_HI; within an ulp of
    the product with the double 0.2 rounded to float."""
    from fractions import Fraction
    lib = oracle_lib()
    c_hi = np.float32(0.2)
    c_lo = np.float32(0.2 - float(c_hi))
    assert c_hi.view(np.uint32) == 0x3E4CCCCD and c_lo.view(np.uint32) == 0xB14CCCCD
    g = seeded_grid(8, 6, 4).astype(np.float32)
    out = g.copy()
    lib.oracle_jacobi2d_f32(out.ctypes.data_as(C.POINTER(C.c_float)), 8, 6, 1, 1)
    for i in range(1, 7):
        for j in range(1, 9):
            s = np.float32(g[i, j]) + np.float32(g[i, j - 1])
            s = np.float32(s + g[i, j + 1])
            s = np.float32(s + g[i - 1, j])
            s = np.float32(s + g[i + 1, j])
            lo = np.float32(s * c_lo)
            want = _round_f32(Fraction(float(s)) * Fraction(float(c_hi)) + Fraction(float(lo)))
            assert out[i, j] == want
            via_double = np.float32(np.float64(s) * 0.2)
            assert abs(int(out[i, j].view(np.int32)) - int(via_double.view(np.int32))) <= 1


def test_residual_matches_numpy():
    lib = oracle_lib()
    g = seeded_grid(20, 10, 2)
    r2 = lib.oracle_residual2_f64(g.ctypes.data_as(C.POINTER(C.c_double)), 20, 10)
    s = (g[1:-1, 1:-1] + g[1:-1, :-2] + g[1:-1, 2:] + g[:-2, 1:-1] + g[2:, 1:-1]) * 0.2
    assert r2 == pytest.approx(float(np.sum((s - g[1:-1, 1:-1]) ** 2)), rel=1e-12)


def test_jacobi1d_known_answer():
    lib = oracle_lib()
    a = np.zeros(10)
    a[:2] = 10.0
    a[-2:] = 10.0
    lib.oracle_jacobi1d_f64(a.ctypes.data_as(C.POINTER(C.c_double)), 6, 1)
    assert a[2] == (10.0 + 10.0 + 0 + 0 + 0) / 5
    assert a[3] == (10.0 + 0 + 0 + 0 + 0) / 5
    assert a[4] == 0.0


def _golden_cases():
    path = os.path.join(GOLDEN, "ref_jacobi2d.json")
    if not os.path.exists(path):
        return []
    with open(path) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["file"])
def test_oracle_matches_reference_kernel_fixture(case):
    """Pin: the oracle reproduces the reference's own jacobi_2d_kernel bit for bit."""
    nx, ny, sweeps, seed = case["nx"], case["ny"], case["sweeps"], case["seed"]
    ref = np.fromfile(os.path.join(GOLDEN, case["file"]), dtype="<f8").reshape(ny + 2, nx + 2)
    out = jac64(seeded_grid(nx, ny, seed), sweeps)
    assert np.array_equal(out.view(np.uint64), ref.view(np.uint64))


def test_golden_fixtures_present():
    assert _golden_cases(), "tests/golden/ref_jacobi2d.json missing (run tests/golden/gen_ref_fixtures.sh on a GPU)"
    assert _golden_cases3(), "tests/golden/ref_jacobi3d.json missing (run tests/golden/gen_ref_fixtures.sh on a GPU)"


def _golden_cases3():
    path = os.path.join(GOLDEN, "ref_jacobi3d.json")
    if not os.path.exists(path):
        return []
    with open(path) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", _golden_cases3(), ids=lambda c: c["file"])
def test_oracle_matches_reference_3d_kernel_fixture(case):
    """Pin: the 3-D oracle reproduces the reference's own jacobi_3d_kernel
    (examples/jacobi-kernel/jacobi_kernel.cu:36-48) bit for bit."""
    from oracle.jacobi import jacobi3d, seeded_grid3d
    nx, ny, nz, sweeps, seed = case["nx"], case["ny"], case["nz"], case["sweeps"], case["seed"]
    ref = np.fromfile(os.path.join(GOLDEN, case["file"]), dtype="<f8").reshape(nz + 2, ny + 2, nx + 2)
    out = jacobi3d(seeded_grid3d(nx, ny, nz, seed), sweeps)
    assert np.array_equal(out.view(np.uint64), ref.view(np.uint64))
    assert np.array_equal(jacobi3d(seeded_grid3d(nx, ny, nz, seed), sweeps, threads=4).view(np.uint64),
                          ref.view(np.uint64))


def test_messaging_cpu_baseline_delivers_everything():
    """The CPU baseline of the messaging benchmarks (oracle/msg_cpu.c)
    delivers every fan-out message on any thread count, and its pingpong
    returns a positive latency."""
    from oracle import msg_cpu
    for threads in (1, 3, 8):
        s, d = msg_cpu.fanout(300, 16, 64, 0xC2, threads)
        assert d == 300 * 16 and s > 0
    assert msg_cpu.pingpong_oneway_s(64, 100) > 0
