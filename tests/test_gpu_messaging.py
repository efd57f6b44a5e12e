"""GPU parity tests of the messaging path against the CPU model (oracle/)."""
import os
import subprocess

import numpy as np
import pytest

from oracle import msgmodel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_hello_chain(rt):
    got = rt.hello()
    assert got.tolist() == msgmodel.hello_chain(rt.n_pes)
    st = rt.last_stats()
    assert st.status == 0
    assert st.delivered == 2 * rt.n_pes


@pytest.mark.parametrize("reversed_order", [False, True])
def test_refnum_order(rt, reversed_order):
    got = rt.refnum(reversed_order)
    assert got == msgmodel.refnum_scenario(reversed_order) == [1, 0]
    st = rt.last_stats()
    assert st.stashed == (1 if reversed_order else 0)


@pytest.mark.parametrize("n,msgs,payload,mode", [
    (64, 4, 16, 0),          # tiny
    (300, 16, 64, 0),        # plain FIFO, more chares than PEs
    (300, 16, 64, 1),        # refnum ladder 0..15
    (4096, 16, 64, 1),       # C2b: 4096 chares x 16 msgs of 64 B, refnums 0..15
    (4096, 16, 64, 0),
    (512, 8, 1024, 1),       # larger payloads
])
def test_fanout_delivery_log(rt, n, msgs, payload, mode):
    seed = 0xC0FFEE + n + mode
    log, ms = rt.fanout(n, msgs, payload, seed, mode)
    chk = msgmodel.check_fanout_log(log, n, msgs, payload, seed, mode)
    assert chk.ok, chk.errors
    assert chk.delivered == n * msgs


def test_fanout_counts_match_model(rt):
    n, msgs, seed = 1000, 16, 7
    log, _ = rt.fanout(n, msgs, 64, seed, 1)
    exp = msgmodel.fanout_expected_counts(n, msgs, seed)
    got = np.zeros_like(exp)
    np.add.at(got, (log[:, 0].astype(np.int64), log[:, 2].astype(np.int64)), 1)
    assert np.array_equal(got, exp)


def test_pingpong_checksums_and_placement(rt):
    sizes = [8, 64, 4096, 65536, 1 << 20]
    rows, sms = rt.pingpong(sizes, round_trips=20, warmup=2, seed=11, verify=True)
    assert sms[0] != sms[1], "pingpong chares must sit on different SMs"
    for r in rows:
        assert r["checksum_errors"] == 0, r
        assert r["oneway_us"] > 0


def _run_ref_example(name, args=(), timeout=120):
    exe = os.path.join(ROOT, "build", "ref_examples", name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (needs the reference tree at build time)")
    env = dict(os.environ, CHARMING_DEADLINE_S="60", CHARMING_IDLE_TIMEOUT_S="3")
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=timeout, env=env)


def test_reference_hello_links_and_runs():
    r = _run_ref_example("hello")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("Hello I'm")]
    n = len(lines)
    assert n > 0 and n % 2 == 0
    for i, line in enumerate(lines):
        assert line == f"Hello I'm {i} of {n}! Received {i}"


def test_reference_refnum_links_and_runs():
    # The reference example never calls end(); the runtime's idle timeout
    # ends the run (status 5) after both messages were delivered in order.
    r = _run_ref_example("refnum")
    assert r.returncode == 5, r.stdout[-2000:] + r.stderr[-2000:]
    got = [l for l in r.stdout.splitlines() if l.startswith("Received message with refnum")]
    assert got == ["Received message with refnum 1", "Received message with refnum 0"]


def test_reference_pingpong_links_and_runs():
    r = _run_ref_example("pingpong", ["8", "4096", "50", "5"])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    sizes = [l for l in r.stdout.splitlines() if l.startswith("Size ")]
    assert [int(l.split()[1]) for l in sizes] == [8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]



def test_gpu_level_program_runs(tmp_path):
    # A program in the reference's GPU-level style (tests/compile/
    # gpu_level_forms.cu, built with -DCHARMING_GPU_LEVEL) gets GPU-level
    # mode from the library's process main: one PE of all blocks, every
    # entry method run by the whole grid, sends collective over the grid.
    arch = "-gencode arch=compute_100a,code=sm_100a"
    lib = os.path.join(ROOT, "charming_b200", "lib", "libcharming.a")
    src = os.path.join(ROOT, "tests", "compile", "gpu_level_forms.cu")
    obj, exe = tmp_path / "glf.o", tmp_path / "glf"
    inc = os.path.join(ROOT, "include")
    r = subprocess.run(f"nvcc -std=c++17 {arch} -rdc=true -DCHARMING_GPU_LEVEL -I{inc} -c {src} -o {obj} && "
                       f"nvcc {arch} -rdc=true -Xnvlink -suppress-stack-size-warning -o {exe} {obj} {lib} -lcudart",
                       shell=True, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    env = dict(os.environ, CHARMING_DEADLINE_S="60", CHARMING_IDLE_TIMEOUT_S="3")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "GPU-level mode: 1 PE of" in r.stdout
    assert "gpu-level forms: pe 0 of 1, rounds 6, hits 3, bad 0" in r.stdout, r.stdout[-2000:]
