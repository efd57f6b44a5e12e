"""GPU tests of the multi-GPU transport (one NVSwitch domain, no relay PE) on
one B200: the PEs of the launch form 2 to 8 GPUs, each with its own inbox
memory and control words, reached through the per-GPU table with
system-scope ticket atomics, sequence words and heads -- the path a PE on one
GPU takes into another GPU's rings over NVLink, with its own memory behind
the pointers. (A run of several processes, one per GPU, maps the peers'
regions with CUDA IPC instead; with one GPU per test run that part is
checked on the CPU, tests/test_multi_gpu_cpu.py.)

Reference: the multi-GPU CE relay (src/comm/get/get.cu:518-690, :783-862;
src/sched/scheduler.cu:78-163). Results are checked against the same CPU
models as on one GPU (oracle/msgmodel.py, the Jacobi oracle). Each case runs
in a child process, so the session's runtime keeps its single-GPU defaults."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def child(code, env=None, timeout=600):
    e = dict(os.environ, **(env or {}))
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=timeout, env=e)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


MESSAGING = """
import json, numpy as np
from charming_b200.runtime import Runtime
from oracle import msgmodel
rt = Runtime(virtual_devs={v}, n_pes={n})
res = dict(n_devs=rt.info["n_devs"], n_pes=rt.n_pes)
res["hello"] = rt.hello().tolist() == msgmodel.hello_chain(rt.n_pes)
res["refnum"] = [rt.refnum(False), rt.refnum(True)]
fan = []
for (n, msgs, payload, mode) in [(300, 16, 64, 0), (300, 16, 64, 1), (4096, 16, 64, 1), (512, 8, 1024, 1)]:
    seed = 0x5EED + n + mode
    log, ms = rt.fanout(n, msgs, payload, seed, mode)
    chk = msgmodel.check_fanout_log(log, n, msgs, payload, seed, mode)
    fan.append([bool(chk.ok), int(chk.delivered) == n * msgs, chk.errors[:3]])
res["fanout"] = fan
rows, sms = rt.pingpong([8, 4096, 1 << 20], round_trips=50, warmup=5, seed=3, verify=True)
res["pingpong_errors"] = sum(r["checksum_errors"] for r in rows)
res["oneway_us_8B"] = rows[0]["oneway_us"]
st = rt.last_stats()
res["status"] = st.status
rt.fini()
print(json.dumps(res))
"""


@pytest.mark.parametrize("vdevs,n_pes", [(2, 148), (4, 148), (8, 144)])
def test_virtual_gpus_messaging_matches_model(vdevs, n_pes):
    """Hello chain, refnum scenario (chare 1 on PE n/2: another GPU),
    fan-out logs (FIFO and refnum ladders, 4096 chares x 16 messages) and
    pingpong checksums across the GPUs' rings (8 GPUs of 18 PEs: 144 of the
    148 SMs)."""
    out = child(MESSAGING.format(v=vdevs, n=n_pes))
    assert out["n_devs"] == vdevs and out["n_pes"] == n_pes
    assert out["hello"]
    assert out["refnum"] == [[1, 0], [1, 0]]
    for ok, complete, errors in out["fanout"]:
        assert ok and complete, errors
    assert out["pingpong_errors"] == 0 and out["status"] == 0
    assert out["oneway_us_8B"] > 0


JACOBI = """
import json, numpy as np
from charming_b200.runtime import Runtime
from charming_b200.jacobi import Jacobi2D, Problem
from oracle import jacobi as oj
rt = Runtime(virtual_devs={v})
same = []
for (nx, ny, px, py, sweeps, depth) in [(333, 201, 5, 3, 37, 6), (1000, 77, 7, 2, 9, 1), (700, 610, 0, 0, 24, 0)]:
    g = oj.seeded_grid(nx, ny, nx + ny)
    with Jacobi2D([Problem(nx, ny, sweeps, px=px, py=py)], depth=depth) as j:
        j.load(0, g)
        j.run()
        out = j.store(0)
    ref = oj.jacobi2d(g.copy(), sweeps)
    same.append(bool(np.array_equal(out.view(np.uint64), ref.view(np.uint64))))
rt.fini()
print(json.dumps(same))
"""


@pytest.mark.parametrize("vdevs", [2, 4])
def test_virtual_gpus_jacobi2d_bit_exact(vdevs):
    """The Jacobi2d chares spread over the GPUs: every halo between chares
    on different GPUs crosses the multi-GPU path; the result is bit for bit
    the oracle's (FP64, depths 6 and 1, explicit and automatic splits)."""
    assert child(JACOBI.format(v=vdevs)) == [True, True, True]


def test_virtual_gpus_idle_timeout_stops_every_gpu():
    """A wait nobody satisfies: PE 0 finds nothing delivered on any GPU for
    the (1 s) idle timeout and stops all of them; the run returns the status
    and the next run on the same runtime is clean."""
    out = child(
        "import json\n"
        "from charming_b200.runtime import Runtime\n"
        "rt = Runtime(virtual_devs=2)\n"
        "st, order = rt.async_wait_chain(40, broken=True)\n"
        "st2, order2 = rt.async_wait_chain(40)\n"
        "print(json.dumps([st, order, st2, order2]))\n",
        env={"CHARMING_IDLE_TIMEOUT_S": "1"})
    st, order, st2, order2 = out
    assert st == 5  # CHARMING_ERR_IDLE_TIMEOUT
    assert order == list(range(39)) + [-1]
    assert st2 == 0 and order2 == list(range(40))


def _ref_example(name, args=(), vdevs=2):
    exe = os.path.join(ROOT, "build", "ref_examples", f"{name}_multi")
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (needs the reference tree at build time)")
    env = dict(os.environ, CHARMING_DEADLINE_S="60", CHARMING_IDLE_TIMEOUT_S="3",
               CHARMING_VIRTUAL_DEVS=str(vdevs))
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=120, env=env)


def test_reference_examples_over_virtual_gpus():
    """The reference's own programs, linked unchanged against the
    multi-GPU build of the library, over 2 GPUs. hello: the chain crosses from the first GPU's PEs to the
    second's, and end() on the second stops the first. refnum: chare 1 on
    PE n/2 (the second GPU) receives in refnum order; the example never
    calls end(), so PE 0 ends the run at the idle timeout (status 5) on
    both GPUs. pingpong: every size between PE 0 and PE n/2."""
    r = _ref_example("hello")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "on 2 GPUs" in r.stdout
    lines = [l for l in r.stdout.splitlines() if l.startswith("Hello I'm")]
    n = len(lines)
    assert n == 2 * 148
    for i, line in enumerate(lines):
        assert line == f"Hello I'm {i} of {n}! Received {i}"
    r = _ref_example("refnum")
    assert r.returncode == 5, r.stdout[-2000:] + r.stderr[-2000:]
    got = [l for l in r.stdout.splitlines() if l.startswith("Received message with refnum")]
    assert got == ["Received message with refnum 1", "Received message with refnum 0"]
    r = _ref_example("pingpong", ["8", "4096", "50", "5"])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    sizes = [l for l in r.stdout.splitlines() if l.startswith("Size ")]
    assert [int(l.split()[1]) for l in sizes] == [8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


IPC_RANK = """
import json, sys
import torch.distributed as dist
rank, port = int(sys.argv[1]), sys.argv[2]
dist.init_process_group("gloo", rank=rank, world_size=2, init_method="tcp://127.0.0.1:" + port)
from charming_b200.runtime import Runtime
rt = Runtime(group=dist.group.WORLD, n_pes=16, ring_bytes=1 << 16, max_msg_bytes=4096,
             stash_bytes=1 << 20, heap_bytes=64 << 20)
info = dict(rt.info)
rt.fini()
dist.destroy_process_group()
print(json.dumps({k: info[k] for k in ("n_pes", "n_blocks", "n_devs", "my_dev")}))
"""


def test_two_processes_export_and_map_inbox_regions():
    """The host side of a run over two processes, on the one GPU this test
    run has: each exports its inbox region with CUDA IPC, the handles go
    through the Python host's allgather (torch.distributed, gloo), each maps
    the other's region, and fini unmaps and frees them between barriers.
    No run is launched: scheduler kernels of two processes that wait on one
    another must not share one GPU (the transport itself is run on one GPU
    by the virtual-GPU tests above, and across processes on the CPU)."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [subprocess.Popen([sys.executable, "-c", IPC_RANK, str(r), str(port)], cwd=ROOT,
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for r in range(2)]
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=300)
        assert p.returncode == 0, o[-2000:] + e[-3000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for rank, info in enumerate(outs):
        assert info == {"n_pes": 32, "n_blocks": 16, "n_devs": 2, "my_dev": rank}
