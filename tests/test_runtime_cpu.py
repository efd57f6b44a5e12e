"""CPU check of the runtime itself: charming_b200/csrc/runtime.cu (scheduler
loop, inbox rings, stash and revive, termination) and the message programs
compiled for the host (tests/emu/rt_emu.cpp). Three builds: one host thread
per PE under AddressSanitizer/UBSan and under ThreadSanitizer (many PEs,
small rings that wrap), and one PE block of many threads under
ThreadSanitizer with call-site-checked barriers and lockstep warps (the
block-collective paths). Delivery logs are checked against the CPU model of
the reference semantics (oracle/msgmodel.py): counts, per-pair order, the
refnum ladder and payload checksums."""
import os
import subprocess

import numpy as np
import pytest

from oracle import msgmodel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "build", "emu")


@pytest.fixture(scope="module")
def emus():
    r = subprocess.run(["make", "-s"], cwd=os.path.join(ROOT, "tests", "emu"), capture_output=True,
                       text=True)
    if r.returncode != 0:
        pytest.fail(r.stdout[-3000:] + r.stderr[-3000:])
    return {k: os.path.join(OUT, k) for k in ("rt_emu", "rt_emu_tsan", "rt_emu_mt")}


def run(exe, args, threads=1, timeout=600):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0", TSAN_OPTIONS="halt_on_error=1",
               RT_EMU_THREADS=str(threads))
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True,
                       timeout=timeout, env=env)
    assert "ThreadSanitizer" not in r.stderr and "divergence" not in r.stderr, r.stderr[-3000:]
    assert "runtime error" not in r.stderr, r.stderr[-3000:]
    return r


def fanout(exe, n_pes, ring, n, msgs, payload, seed, mode, threads=1):
    r = run(exe, ["fanout", n_pes, ring, n, msgs, payload, seed, mode], threads)
    head = r.stdout.splitlines()[0]
    assert r.returncode == 0 and head.startswith("status=0"), (head, r.stderr[-2000:])
    rows = [l.split()[1:] for l in r.stdout.splitlines() if l.startswith("L ")]
    log = np.array([[int(x, 16) for x in row] for row in rows], dtype=np.uint32).reshape(-1, 8)
    chk = msgmodel.check_fanout_log(log, n, msgs, payload, seed, mode)
    assert chk.ok, chk.errors
    assert chk.delivered == n * msgs
    return int(head.split("deferred=")[1].split()[0])


@pytest.mark.parametrize("n_pes,ring,n,msgs,payload,mode", [
    (16, 65536, 300, 16, 64, 0),      # rings wrap many times
    (16, 262144, 300, 16, 64, 1),     # refnum ladder through the stash
    (32, 1 << 20, 4096, 16, 64, 1),   # the C2b shape on 32 PEs
    (24, 1 << 20, 512, 8, 1024, 1),   # larger payloads, stash arena use
])
def test_fanout_many_pes(emus, n_pes, ring, n, msgs, payload, mode):
    fanout(emus["rt_emu"], n_pes, ring, n, msgs, payload, 0xC0FFEE + n + mode, mode)


@pytest.mark.parametrize("n_pes,ring,n,msgs,payload,mode", [
    (8, 65536, 200, 8, 64, 1),
    (8, 65536, 120, 8, 64, 0),
])
def test_fanout_many_pes_threads_race_free(emus, n_pes, ring, n, msgs, payload, mode):
    fanout(emus["rt_emu_tsan"], n_pes, ring, n, msgs, payload, 7 + mode, mode)


@pytest.mark.parametrize("threads", [32, 96])
@pytest.mark.parametrize("n,msgs,payload,mode,ring", [
    (32, 16, 64, 1, 1 << 18),
    (40, 8, 1024, 1, 1 << 20),
    (48, 8, 256, 0, 1 << 18),
])
def test_fanout_block_collective_paths(emus, threads, n, msgs, payload, mode, ring):
    fanout(emus["rt_emu_mt"], 1, ring, n, msgs, payload, 0xC0FFEE, mode, threads)


@pytest.mark.parametrize("threads", [64, 128])
@pytest.mark.parametrize("n,msgs,payload,mode,ring", [
    (40, 16, 64, 0, 1 << 18),     # FIFO: nearly every delivery in a batch
    (40, 16, 64, 1, 1 << 18),     # refnum ladders: a mismatch ends a batch
    (16, 8, 256, 1, 2048),        # tiny ring: batches over wrapped tickets, deferred sends
])
def test_warp_entry_methods_run_in_batches(emus, threads, n, msgs, payload, mode, ring):
    """The fan-out's receive is a warp-level entry method: warp 0 scans the
    cells after the head message and the block runs up to one delivery per
    warp at once (2 and 4 warps, lockstep, ThreadSanitizer). The log must
    still match the model exactly (per-pair order, refnum ladders)."""
    r = run(emus["rt_emu_mt"], ["fanout", 1, ring, n, msgs, payload, 0xBA7 + n + mode, mode], threads)
    head = r.stdout.splitlines()[0]
    assert r.returncode == 0 and head.startswith("status=0"), (head, r.stderr[-2000:])
    rows = [l.split()[1:] for l in r.stdout.splitlines() if l.startswith("L ")]
    log = np.array([[int(x, 16) for x in row] for row in rows], dtype=np.uint32).reshape(-1, 8)
    chk = msgmodel.check_fanout_log(log, n, msgs, payload, 0xBA7 + n + mode, mode)
    assert chk.ok, chk.errors
    assert int(head.split("batched=")[1].split()[0]) > 0


@pytest.mark.parametrize("exe,n_pes,threads,ring,n,msgs,payload,mode", [
    # every PE's start entry methods send far more than the receivers'
    # rings hold, to PEs that are doing the same: each send that finds no
    # space moves to the sender's outbox, the entry method returns, and the
    # scheduler loop copies it into the ring later (before: RING_FULL)
    ("rt_emu", 8, 1, 2048, 64, 16, 256, 0),
    ("rt_emu", 4, 1, 2048, 8, 16, 1024, 1),
    ("rt_emu_tsan", 8, 1, 2048, 64, 8, 256, 1),
    ("rt_emu_mt", 1, 32, 2048, 16, 8, 256, 1),   # one PE sending to itself
])
def test_full_rings_defer_sends_instead_of_deadlock(emus, exe, n_pes, threads, ring, n, msgs, payload,
                                                   mode):
    deferred = fanout(emus[exe], n_pes, ring, n, msgs, payload, 0xDEF + n, mode, threads)
    assert deferred > 0


@pytest.mark.parametrize("reversed_order", [0, 1])
@pytest.mark.parametrize("exe,n_pes,threads", [("rt_emu", 6, 1), ("rt_emu_mt", 1, 64)])
def test_refnum_scenario(emus, exe, n_pes, threads, reversed_order):
    r = run(emus[exe], ["refnum", n_pes, 65536, reversed_order], threads)
    assert r.returncode == 0
    out = r.stdout.split("out=")[1].split(",")
    assert [int(out[0]), int(out[1])] == msgmodel.refnum_scenario(bool(reversed_order)) == [1, 0]


@pytest.mark.parametrize("exe,n_pes,threads", [("rt_emu", 5, 1), ("rt_emu_mt", 1, 32)])
def test_hello_chain(emus, exe, n_pes, threads):
    r = run(emus[exe], ["hello", n_pes, 65536], threads)
    assert r.returncode == 0
    out = [int(x) for x in r.stdout.split("out=")[1].strip().strip(",").split(",")]
    assert out[: 2 * n_pes] == list(range(2 * n_pes))


@pytest.mark.parametrize("exe,n_pes,threads,n", [
    ("rt_emu", 4, 1, 12), ("rt_emu_tsan", 6, 1, 18), ("rt_emu_mt", 1, 64, 5)])
def test_async_wait_chain(emus, exe, n_pes, threads, n):
    """Chare i's entry method runs once its two signal words are >= 1, which
    chare i-1 sets when it runs: the wake order is the chain order, and
    several waits are pending per PE at once."""
    r = run(emus[exe], ["await", n_pes, 65536, n, 0], threads)
    out = r.stdout.strip().split("order=")
    assert out[0].strip() == "status=0", r.stdout + r.stderr[-2000:]
    assert [int(x) for x in out[1].strip(",").split(",")] == list(range(n))


@pytest.mark.parametrize("exe,n_pes,threads,n", [
    ("rt_emu", 6, 1, 18), ("rt_emu_tsan", 3, 1, 9), ("rt_emu_mt", 1, 64, 5)])
def test_async_wait_never_satisfied_ends_at_idle_timeout(emus, exe, n_pes, threads, n):
    """Nobody signals the last chare: its wait runs out at the idle timeout
    (1 s here) and the run returns that error status; the others woke in
    order."""
    r = run(emus[exe], ["await", n_pes, 65536, n, 1], threads, timeout=120)
    out = r.stdout.strip().split("order=")
    assert out[0].strip() == "status=5", r.stdout + r.stderr[-2000:]
    assert [int(x) for x in out[1].strip(",").split(",")] == list(range(n - 1)) + [-1]


@pytest.mark.parametrize("exe,n_pes,threads,n,blocks,rounds", [
    ("rt_emu", 4, 1, 8, 8, 60),       # heaps of 64 KiB wrap many times
    ("rt_emu_tsan", 4, 1, 8, 5, 60),
    ("rt_emu_mt", 1, 64, 3, 8, 20),
])
def test_user_heap(emus, exe, n_pes, threads, n, blocks, rounds):
    """malloc_user / free_user: blocks keep their contents until freed,
    space comes back after out-of-order frees (more bytes are taken over
    the run than the heap holds), and a block is readable from another
    PE."""
    r = run(emus[exe], ["userheap", n_pes, 65536, n, blocks, rounds, 5], threads)
    f = dict(kv.split("=") for kv in r.stdout.split())
    assert f["status"] == "0", r.stdout + r.stderr[-2000:]
    assert int(f["bad"]) == 0
    assert int(f["taken"]) == int(f["freed"]) and int(f["failed"]) == 0
    assert int(f["checked"]) == n and int(f["done"]) == n
    # the PEs took several times their 64 KiB heaps over the run
    assert int(f["bytes"]) > 3 * n_pes * 65536


@pytest.mark.parametrize("exe,n_pes,threads,n,nx,ny,iters,mode", [
    ("rt_emu", 5, 1, 5, 16, 30, 7, 0),      # signals, one chare per PE, waits in the entry method
    ("rt_emu", 3, 1, 7, 16, 40, 9, 1),      # signals, async_wait, several chares per PE
    ("rt_emu", 3, 1, 7, 20, 33, 9, 2),      # rows as messages tagged with refnums
    ("rt_emu", 1, 1, 3, 12, 20, 6, 2),      # every neighbour on the same PE
    ("rt_emu_tsan", 4, 1, 6, 16, 30, 5, 1),
    ("rt_emu_tsan", 4, 1, 6, 16, 30, 5, 2),
    ("rt_emu_mt", 1, 64, 4, 136, 24, 5, 1),  # warps walking column strips
    ("rt_emu_mt", 1, 32, 4, 64, 24, 5, 2),
])
def test_decomp1d_matches_oracle(emus, exe, n_pes, threads, n, nx, ny, iters, mode):
    """jacobi2d-decomp1d on the real scheduler, bit for bit against the CPU
    restatement (oracle/jacobi_oracle.c oracle_decomp1d_f32)."""
    from oracle import jacobi as oj
    r = run(emus[exe], ["decomp1d", n_pes, 65536, n, nx, ny, iters, mode], threads)
    lines = r.stdout.splitlines()
    assert lines and lines[0] == "status=0", (lines[:2], r.stderr[-2000:])
    got = np.array([[int(x, 16) for x in l.split()[1:]] for l in lines if l.startswith("G ")], dtype=np.uint32)
    ref = oj.decomp1d(n, nx, ny, iters)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref.view(np.uint32))


@pytest.mark.parametrize("exe,blocks,n,nx,ny,iters,mode", [
    ("rt_emu", 4, 1, 64, 40, 5, 0),        # one chare, its own neighbour both ways
    ("rt_emu", 4, 1, 64, 40, 5, 1),
    ("rt_emu", 4, 1, 64, 40, 5, 2),
    ("rt_emu", 3, 3, 64, 30, 4, 1),        # several chares on the one PE
    ("rt_emu", 5, 2, 40, 50, 6, 2),
    ("rt_emu_tsan", 4, 1, 64, 40, 5, 1),   # the blocks' hand-offs under ThreadSanitizer
    ("rt_emu_tsan", 3, 3, 64, 30, 4, 2),
])
def test_gpu_level_decomp1d_matches_oracle(emus, exe, blocks, n, nx, ny, iters, mode):
    """GPU-level mode on the real scheduler: `blocks` emulated blocks form
    PE 0; block 0 schedules, every block runs each entry method and each
    collective send (group_state hand-offs and grid barriers)."""
    from oracle import jacobi as oj
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0", TSAN_OPTIONS="halt_on_error=1",
               RT_EMU_THREADS="1", RT_EMU_GPU_LEVEL="1")
    r = subprocess.run([emus[exe], "decomp1d", str(blocks), "65536", str(n), str(nx), str(ny), str(iters),
                        str(mode)], capture_output=True, text=True, timeout=600, env=env)
    assert "ThreadSanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-3000:]
    lines = r.stdout.splitlines()
    assert lines and lines[0] == "status=0", (lines[:2], r.stderr[-2000:])
    got = np.array([[int(x, 16) for x in l.split()[1:]] for l in lines if l.startswith("G ")], dtype=np.uint32)
    ref = oj.decomp1d(n, nx, ny, iters)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref.view(np.uint32))


def serve(exe, n_pes, n_req, seed, wpp, max_inflight, side, dtype, threads=1, ring=65536):
    """Solve server on the CPU: the real scheduler runs the Jacobi2d chares
    in serving mode (apps/jacobi2d.cu) and admission runs apps/serve_host.h;
    a host thread submits seeded requests of mixed sizes while others run
    and compares every result bit for bit with the serial oracle."""
    r = run(exe, ["serve", n_pes, ring, n_req, seed, wpp, max_inflight, side, dtype], threads, timeout=900)
    lines = r.stdout.splitlines()
    assert r.returncode == 0 and lines and "bad=0" in lines[-1], (lines[-5:], r.stderr[-2000:])
    results = [l for l in lines if l.startswith("R ")]
    refused = [l for l in lines if l.startswith("S ")]
    assert len(results) + len(refused) == n_req
    assert all("same=1" in l for l in results)
    # workers and slots were reused: more requests than slots completed
    assert len(results) > max_inflight
    return results


@pytest.mark.parametrize("exe,n_pes,threads,n_req,dtype,seed,ring", [
    ("rt_emu", 6, 1, 40, 0, 7, 65536),        # ASan + UBSan, FP64
    ("rt_emu", 6, 1, 40, 1, 8, 65536),        # FP32 sweeps, FP64 residual
    ("rt_emu_tsan", 8, 1, 30, 1, 11, 65536),  # PE threads under ThreadSanitizer
    ("rt_emu_mt", 1, 64, 10, 0, 5, 65536),    # one PE block of 64 threads
    ("rt_emu_mt", 1, 64, 10, 0, 5, 4096),     # and with rings that fill up
])
def test_serving_results_match_oracle(emus, exe, n_pes, threads, n_req, dtype, seed, ring):
    wpp = 6 if n_pes == 1 else 3
    serve(emus[exe], n_pes, n_req, seed, wpp, 4, 16, dtype, threads, ring=ring)


@pytest.mark.parametrize("exe,n_pes,threads", [("rt_emu", 4, 1), ("rt_emu_mt", 1, 32)])
def test_server_nobody_stops_ends_at_deadline(emus, exe, n_pes, threads):
    # the server chare calls itself forever; the busy PE must still see the
    # run deadline (1 s here) and the run must end with DEADLINE
    r = run(emus[exe], ["serve", n_pes, 65536, -1, 1, 2, 4, 16, 0], threads, timeout=120)
    assert r.returncode == 0 and "status=6" in r.stdout, (r.stdout[-500:], r.stderr[-1500:])


def test_serve_host_logic():
    """Slab allocator, FIFO admission against budget / slots / workers,
    balanced worker placement, generations and staged descriptors
    (tests/emu/serve_host_test.cpp on apps/serve_host.h)."""
    r = subprocess.run(["make", "-s", os.path.join("..", "..", "build", "emu", "serve_host_test")],
                       cwd=os.path.join(ROOT, "tests", "emu"), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    r = run(os.path.join(OUT, "serve_host_test"), [])
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr[-2000:]
