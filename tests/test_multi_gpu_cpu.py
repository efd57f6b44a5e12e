"""CPU check of the multi-GPU transport (runtime.cu with several GPUs, one
NVSwitch domain): the runtime compiled for the host (tests/emu/rt_emu.cpp)
in its two multi-GPU forms.

* Virtual GPUs: the PE blocks of one process form n GPUs, each with its own
  inbox memory and control words, addressed through the per-GPU table with
  system-scope atomics -- the code path that runs on one B200.
* Several processes: w emulator processes, one GPU each, whose inbox sides
  are files that every process maps shared (in the role of CUDA IPC over
  NVLink), bootstrapped by the process main's file rendezvous
  (charming_b200/csrc/rendezvous.h). A sender's ticket atomic, payload
  stores and release store land in another process's memory, as they land
  in another GPU's over NVLink.

Delivery logs are checked against the CPU model of the reference semantics
(oracle/msgmodel.py), as for one GPU. The reference's multi-GPU path is its
CE relay over NVSHMEM (src/comm/get/get.cu:518-690, :783-862; src/sched/
scheduler.cu:78-163): the observable semantics -- global PE numbering,
placement, per-pair order, refnum matching, termination -- are the same."""
import os
import subprocess
import tempfile

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
    return {k: os.path.join(OUT, k) for k in ("rt_emu", "rt_emu_tsan")}


def _env(**extra):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0", TSAN_OPTIONS="halt_on_error=1",
               RT_EMU_THREADS="1")
    env.update({k: str(v) for k, v in extra.items()})
    return env


def _check(r):
    assert "ThreadSanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-3000:]
    assert "AddressSanitizer" not in r.stderr, r.stderr[-3000:]


def run_virtual(exe, vdevs, args, timeout=600):
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout,
                       env=_env(RT_EMU_VDEVS=vdevs))
    _check(r)
    return r


def run_world(exe, world, args, timeout=300):
    """The same command as `world` processes, one emulated GPU each."""
    with tempfile.TemporaryDirectory() as d:
        procs = [subprocess.Popen([exe] + [str(a) for a in args], stdout=subprocess.PIPE,
                                  stderr=subprocess.PIPE, text=True,
                                  env=_env(RT_EMU_WORLD=world, RT_EMU_RANK=r, RT_EMU_DIR=d))
                 for r in range(world)]
        outs = []
        for p in procs:
            try:
                o, e = p.communicate(timeout=timeout)
            except subprocess.TimeoutExpired:
                for q in procs:
                    q.kill()
                raise
            outs.append(subprocess.CompletedProcess(p.args, p.returncode, o, e))
    for r in outs:
        _check(r)
    return outs


def parse_fanout(r):
    lines = r.stdout.splitlines()
    head = dict(kv.split("=") for kv in lines[0].split())
    rows = [l.split()[1:] for l in lines if l.startswith("L ")]
    log = np.array([[int(x, 16) for x in row] for row in rows], dtype=np.uint32).reshape(-1, 8)
    return head, log


def check_log(log, n, msgs, payload, seed, mode):
    chk = msgmodel.check_fanout_log(log, n, msgs, payload, seed, mode)
    assert chk.ok, chk.errors[:10]
    assert chk.delivered == n * msgs


# ---- virtual GPUs (one process, one launch) ----------------------------------

@pytest.mark.parametrize("exe,vdevs,n_pes,ring,n,msgs,payload,mode", [
    ("rt_emu", 2, 8, 65536, 200, 16, 64, 0),     # rings wrap; cross-GPU and local sends
    ("rt_emu", 4, 16, 262144, 300, 16, 64, 1),   # refnum ladder through the stash
    ("rt_emu", 8, 16, 1 << 20, 512, 8, 1024, 1), # eight GPUs of two PEs
    ("rt_emu", 2, 8, 2048, 64, 16, 256, 0),      # full rings: sends deferred to the outbox
    ("rt_emu_tsan", 2, 8, 65536, 120, 8, 64, 1),
])
def test_virtual_gpus_fanout(emus, exe, vdevs, n_pes, ring, n, msgs, payload, mode):
    seed = 0xD15 + n + mode
    r = run_virtual(emus[exe], vdevs, ["fanout", n_pes, ring, n, msgs, payload, seed, mode])
    head, log = parse_fanout(r)
    assert r.returncode == 0 and head["status"] == "0", (r.stdout[:300], r.stderr[-2000:])
    check_log(log, n, msgs, payload, seed, mode)
    # one process: the chares' shared counter saw every receiving chare
    assert int(head["chares_done"]) == len({int(r[0]) for r in log})


@pytest.mark.parametrize("vdevs,n_pes", [(2, 4), (4, 8)])
def test_virtual_gpus_hello_and_refnum(emus, vdevs, n_pes):
    r = run_virtual(emus["rt_emu"], vdevs, ["hello", n_pes, 65536])
    assert r.returncode == 0
    out = [int(x) for x in r.stdout.split("out=")[1].strip().strip(",").split(",")]
    assert out[: 2 * n_pes] == list(range(2 * n_pes))
    for rev in (0, 1):  # chare 1 lives on PE n/2: another GPU
        r = run_virtual(emus["rt_emu"], vdevs, ["refnum", n_pes, 65536, rev])
        assert r.returncode == 0
        out = r.stdout.split("out=")[1].split(",")
        assert [int(out[0]), int(out[1])] == msgmodel.refnum_scenario(bool(rev))


# ---- several processes (one GPU each, inbox sides mapped shared) ---------------

@pytest.mark.parametrize("world,pes", [(2, 3), (3, 2), (4, 2)])
def test_processes_hello_chain(emus, world, pes):
    """2 * n_pes chares, each forwarding value + 1 to the next: the chain
    crosses every process; the last chare's end() stops all of them."""
    outs = run_world(emus["rt_emu"], world, ["hello", pes, 65536])
    n = 2 * pes * world
    merged = np.full(n, -1)
    for r in outs:
        assert r.returncode == 0 and r.stdout.startswith("status=0"), (r.stdout[:200], r.stderr[-2000:])
        vals = np.array([int(x) for x in r.stdout.split("out=")[1].strip().strip(",").split(",")][:n])
        mine = vals >= 0
        assert (merged[mine] == -1).all()  # each chare on exactly one process
        merged[mine] = vals[mine]
    assert merged.tolist() == list(range(n))


@pytest.mark.parametrize("rev", [0, 1])
def test_processes_refnum(emus, rev):
    """Chare 0 on process 0, chare 1 on PE n/2 (process 1): the early
    message waits in process 1's stash until its refnum matches."""
    outs = run_world(emus["rt_emu"], 2, ["refnum", 2, 65536, rev])
    got = None
    for r in outs:
        assert r.returncode == 0, r.stderr[-2000:]
        vals = [int(x) for x in r.stdout.split("out=")[1].split(",")[:2]]
        if vals != [-1, -1]:
            got = vals
    assert got == msgmodel.refnum_scenario(bool(rev))


@pytest.mark.parametrize("world,pes,ring,n,msgs,payload,mode,reps", [
    (2, 4, 65536, 200, 16, 64, 0, 1),     # rings wrap many times
    (2, 4, 262144, 160, 16, 64, 1, 2),    # refnums; two runs in a row
    (3, 3, 1 << 20, 240, 8, 1024, 1, 1),  # larger payloads, three GPUs
    (2, 4, 2048, 48, 16, 256, 0, 1),      # full rings: deferred sends cross processes
])
def test_processes_fanout(emus, world, pes, ring, n, msgs, payload, mode, reps):
    """Every chare sends to seeded destinations anywhere in the run; each
    process logs the deliveries to its own chares (the other records stay
    zero), and the merged log must match the model exactly."""
    seed = 0xAB + n + mode
    outs = run_world(emus["rt_emu"], world, ["fanout", pes, ring, n, msgs, payload, seed, mode, reps])
    merged = None
    done = 0
    for r in outs:
        head, log = parse_fanout(r)
        assert r.returncode == 0 and head["status"] == "0", (r.stdout[:300], r.stderr[-2000:])
        merged = log if merged is None else merged | log
        done += int(head["chares_done"])
    check_log(merged, n, msgs, payload, seed, mode)
    # chare 0's process counted the completion messages of every receiving chare
    assert done == len({int(r[0]) for r in merged})


def test_processes_idle_timeout_reaches_every_gpu(emus):
    """A program that never calls end(): PE 0 (process 0) finds nothing
    delivered anywhere for the idle timeout and stops the run; the other
    process ends with the same status and the PE that recorded it."""
    outs = run_world(emus["rt_emu"], 2, ["fanout", 2, 65536, 16, 4, 64, 3, 0, 1, 1], timeout=120)
    for r in outs:
        head, _ = parse_fanout(r)
        assert head["status"] == "5", (r.stdout[:200], r.stderr[-1000:])  # CHARMING_ERR_IDLE_TIMEOUT
        assert head["err_pe"] == "0"


# ---- the Python host's collectives (torch.distributed, gloo) -------------------

def _collectives_rank(rank, world, port, q):
    import ctypes as C
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    from charming_b200.runtime import host_collectives
    ag, bar = host_collectives()
    mine = (C.c_ubyte * 72)(*[(rank * 31 + i) & 255 for i in range(72)])
    out = (C.c_ubyte * (72 * world))()
    rc = ag(None, C.cast(mine, C.c_void_p), C.cast(out, C.c_void_p), 72)
    rc2 = bar(None)
    q.put((rank, rc, rc2, bytes(out)))
    dist.destroy_process_group()


def test_python_host_collectives_over_gloo():
    """The allgather and barrier that charming_init_devices calls back into
    (here called through their ctypes function pointers, as the library
    does): every rank gets every rank's record in rank order."""
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 2
    ps = [ctx.Process(target=_collectives_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
    want = b"".join(bytes((r * 31 + i) & 255 for i in range(72)) for r in range(world))
    for rank, rc, rc2, out in got:
        assert rc == 0 and rc2 == 0
        assert out == want
