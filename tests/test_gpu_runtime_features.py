"""GPU tests of the runtime features beyond plain invoke: async_wait
(reference include/chare.h:214-239, src/comm/get/get.cu:1172-1202),
malloc_user / free_user (include/charming.h:33-34, get.cu:1348-1362), and
sends that find their destination ring full (the outbox). Runs that need a
non-default configuration (short idle timeout, small rings) go to a child
process, so the session's runtime keeps its defaults."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import msgmodel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def child(code, env=None, timeout=300):
    e = dict(os.environ, **(env or {}))
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=timeout, env=e)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_async_wait_chain_wakes_in_order(rt):
    n = 3 * rt.n_pes  # several waits pending on every PE at once
    status, order = rt.async_wait_chain(n)
    assert status == 0
    assert order == list(range(n))


def test_async_wait_never_satisfied_ends_with_idle_timeout():
    # nobody signals the last chare: its wait runs out at the (1 s) idle
    # timeout, the run returns that status and the device stays usable
    out = child(
        "import json\n"
        "from charming_b200 import runtime\n"
        "rt = runtime()\n"
        "st, order = rt.async_wait_chain(40, broken=True)\n"
        "st2, order2 = rt.async_wait_chain(40)\n"
        "print(json.dumps([st, order, st2, order2]))\n",
        env={"CHARMING_IDLE_TIMEOUT_S": "1"})
    st, order, st2, order2 = out
    assert st == 5  # CHARMING_ERR_IDLE_TIMEOUT
    assert order == list(range(39)) + [-1]
    assert st2 == 0 and order2 == list(range(40))


def test_user_heap_blocks_reused_and_visible_across_pes(rt):
    n = 2 * rt.n_pes
    out = rt.user_heap_check(n, blocks=8, rounds=300, seed=9)
    assert out["bad"] == 0 and out["failed"] == 0
    assert out["taken"] == out["freed"]
    assert out["checked"] == n and out["done"] == n
    # each PE took more than its 1 MiB heap over the run
    assert out["bytes"] > 2 * rt.n_pes * (1 << 20)


@pytest.mark.parametrize("n,msgs,payload,mode", [(2048, 16, 256, 1), (1024, 8, 1024, 0)])
def test_full_rings_defer_sends(n, msgs, payload, mode):
    # 8 KiB inbox rings: the start entry methods send far more than the
    # rings hold, to PEs doing the same; full rings move sends to the
    # outbox and the run completes with the model's delivery log
    seed = 0xDEF + n
    out = child(
        "import json\n"
        "from charming_b200 import runtime\n"
        "from oracle import msgmodel\n"
        "rt = runtime(ring_bytes=8192, max_msg_bytes=4096)\n"
        f"log, _ = rt.fanout({n}, {msgs}, {payload}, {seed}, {mode})\n"
        "st = rt.last_stats()\n"
        f"chk = msgmodel.check_fanout_log(log, {n}, {msgs}, {payload}, {seed}, {mode})\n"
        "print(json.dumps([chk.ok, chk.delivered, st.deferred, chk.errors[:5]]))\n")
    ok, delivered, deferred, errors = out
    assert ok, errors
    assert delivered == n * msgs
    assert deferred > 0


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_sm_pingpong_floor(rt, mode):
    r = rt.sm_pingpong(mode, round_trips=2000)
    assert r["sm_pair"][0] != r["sm_pair"][1]
    assert 0 < r["oneway_ns"] < 100000


@pytest.mark.parametrize("n,nx,ny,iters,mode", [
    (148, 256, 600, 30, 0),    # signals waited inside the entry method, one chare per PE
    (148, 256, 600, 30, 1),    # async_wait
    (148, 256, 600, 30, 2),    # rows as refnum-tagged messages
    (400, 64, 1203, 17, 1),    # several chares per PE, uneven bands
    (400, 64, 1203, 17, 2),
    (3, 1024, 40, 9, 2),       # neighbours on the same PE
])
def test_decomp1d_matches_oracle(rt, n, nx, ny, iters, mode):
    from oracle import jacobi as oj
    if mode == 0 and n > rt.n_pes:
        pytest.skip("one chare per PE")
    got, _ = rt.decomp1d(n, nx, ny, iters, mode)
    ref = oj.decomp1d(n, nx, ny, iters)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_gpu_level_decomp1d_matches_oracle():
    # GPU-level mode (every block forms PE 0): the decomp1d chares run each
    # entry method on the whole grid; all three ways to meet the neighbours,
    # bit for bit against the oracle. A program that is not written for the
    # mode is refused with a configuration error, and the runtime goes on.
    out = child(
        "import json\n"
        "import numpy as np\n"
        "from charming_b200.runtime import Runtime\n"
        "from charming_b200._lib import CharmingError\n"
        "from oracle import jacobi as oj\n"
        "rt = Runtime(gpu_level=1)\n"
        "res = [rt.n_pes, rt.info['n_blocks'], rt.info['gpu_level']]\n"
        "for n, nx, ny, it, mode in [(1, 1024, 600, 9, 0), (1, 1024, 600, 9, 1), (1, 1024, 600, 9, 2),\n"
        "                            (4, 512, 300, 7, 1), (4, 512, 300, 7, 2), (3, 64, 40, 5, 2),\n"
        "                            (2, 4096, 1000, 4, 1)]:\n"
        "    got, _ = rt.decomp1d(n, nx, ny, it, mode)\n"
        "    ref = oj.decomp1d(n, nx, ny, it)\n"
        "    res.append(bool(np.array_equal(got.view(np.uint32), ref.view(np.uint32))))\n"
        "try:\n"
        "    rt.hello()\n"
        "    res.append('hello ran')\n"
        "except CharmingError as e:\n"
        "    res.append(e.code)\n"
        "got, _ = rt.decomp1d(2, 256, 100, 3, 2)\n"
        "res.append(bool(np.array_equal(got.view(np.uint32), oj.decomp1d(2, 256, 100, 3).view(np.uint32))))\n"
        "print(json.dumps(res))\n")
    n_pes, n_blocks, gl = out[:3]
    assert n_pes == 1 and gl == 1 and n_blocks > 1
    assert out[3:10] == [True] * 7
    assert out[10] == 14  # CHARMING_ERR_CONFIG
    assert out[11] is True


@pytest.mark.parametrize("nx,ny,nz,sweeps,seed", [
    (6, 5, 4, 1, 1), (17, 9, 11, 3, 2), (33, 7, 13, 5, 3),   # the golden fixtures' shapes
    (64, 48, 40, 4, 5),                                     # whole tiles
    (97, 35, 70, 7, 6),                                     # ragged tiles, several z runs
    # even row pitch: the TMA plane-ring kernel
    (32, 16, 9, 4, 9),                                      # exactly one box
    (94, 35, 70, 3, 7),                                     # ragged tiles, several z runs
    (62, 16, 300, 2, 8),                                    # long z runs, more planes than slots
])
def test_jacobi3d_matches_oracle(rt, nx, ny, nz, sweeps, seed):
    from oracle import jacobi as oj
    g = oj.seeded_grid3d(nx, ny, nz, seed)
    got, _ = rt.jacobi3d(g, sweeps)
    ref = oj.jacobi3d(g, sweeps)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
