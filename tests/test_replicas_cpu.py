"""The multi-GPU plumbing of bench.py (replicas only) on CPU: two gloo
ranks join through the torchrun environment, the job's time is the max over
ranks, and the whole-job value sums every rank's work over that time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    dist, r, local, w = bench.dist_setup("gloo")
    assert (r, w) == (rank, world)
    bench.barrier(dist, local)
    ms = bench.dist_max(dist, 10.0 + 5.0 * rank, local)  # rank 1 is the slow one
    value = bench.replica_value(1e9, 4, w, ms)
    out.put((rank, ms, value))
    bench.barrier(dist, local)
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replicas_max_over_ranks_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    for rank, ms, value in res:
        assert ms == 15.0  # every rank sees the slowest rank's time
        assert value == pytest.approx(1e9 * 4 * world / 15e-3 / 1e9)
