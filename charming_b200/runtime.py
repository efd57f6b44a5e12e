"""Host-side interface of the runtime (Python mirror of include/charming_c.h).

The reference's host interface is its process ``main()``
(src/charming.cu:50-263): bootstrap, one launch of the persistent scheduler,
teardown.  ``Runtime`` exposes the same life cycle (``init`` / ``run`` /
``fini``) plus the built-in programs, over the C ABI of
``libcharming_b200.so``.  Every call goes to the GPU; errors raise
``CharmingError`` with the runtime's status code.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check

DEFAULTS = dict(device=0, pes_per_sm=1, threads_per_pe=512, n_pes=0, ring_bytes=4 << 20,
                max_msg_bytes=(1 << 20) + 64, stash_bytes=4 << 20, stash_entries=4096,
                heap_bytes=1 << 30, stack_bytes=8192, deadline_s=120.0, idle_timeout_s=10.0,
                free_chares_at_exit=1, verbose=0)


@dataclass
class RunStats:
    delivered: int
    sent: int
    stashed: int
    revived: int
    bytes_sent: int
    idle_polls: int
    space_waits: int
    kernel_ms: float
    loop_ms: float
    main_ms: float
    status: int
    idle_ms: float = 0.0
    em_ms: float = 0.0
    deferred: int = 0
    ticket_ms: float = 0.0
    space_ms: float = 0.0
    batched: int = 0


def host_collectives(group=None):
    """The allgather and barrier a run over several GPUs needs from its host
    (charming_devices), over a torch.distributed process group (a CPU
    backend such as gloo: they exchange host bytes).  Returns the two ctypes
    callbacks; keep them alive as long as the runtime."""
    import torch
    import torch.distributed as dist

    def allgather(_ctx, mine, out, nbytes):
        try:
            t = torch.frombuffer(bytearray(C.string_at(mine, nbytes)), dtype=torch.uint8)
            parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
            dist.all_gather(parts, t, group=group)
            buf = b"".join(bytes(p.numpy()) for p in parts)
            C.memmove(out, buf, len(buf))
            return 0
        except Exception:  # the C side reports the failure
            return -1

    def barrier(_ctx):
        try:
            dist.barrier(group=group)
            return 0
        except Exception:
            return -1

    return _lib.ALLGATHER_FN(allgather), _lib.BARRIER_FN(barrier)


class Runtime:
    """One initialised runtime on one GPU (process-wide, like the reference).

    Several GPUs: ``group`` (a torch.distributed process group, one rank per
    GPU, a CPU backend) makes a run over all its ranks, collective like the
    reference's NVSHMEM runs; ``virtual_devs=n`` splits this GPU's PEs into n
    GPUs in one launch (the same transport on one GPU). Both load the
    multi-GPU build of the library (one build per process)."""

    _active: "Runtime | None" = None

    def __init__(self, group=None, virtual_devs: int = 1, **overrides):
        self.lib = _lib.load(multi=group is not None or virtual_devs > 1)
        cfg = _lib.Config()
        self.lib.charming_default_config(C.byref(cfg))
        for k, v in overrides.items():
            if not hasattr(cfg, k):
                raise KeyError(f"unknown config field {k}")
            setattr(cfg, k, v)
        if Runtime._active is not None:
            Runtime._active.fini()
        devs = _lib.Devices()
        devs.rank, devs.world, devs.virtual_devs = 0, 1, virtual_devs
        self._callbacks = None
        if group is not None:
            import torch.distributed as dist
            devs.rank, devs.world = dist.get_rank(group), dist.get_world_size(group)
            self._callbacks = host_collectives(group)
            devs.allgather, devs.barrier = self._callbacks
        check(self.lib.charming_init_devices(C.byref(cfg), C.byref(devs)), "charming_init_devices")
        Runtime._active = self
        self.config = cfg
        inf = _lib.Info()
        check(self.lib.charming_get_info(C.byref(inf)), "charming_get_info")
        self.info = {f: getattr(inf, f) for f, _ in _lib.Info._fields_}

    # ---- life cycle --------------------------------------------------------
    def fini(self) -> None:
        if Runtime._active is self:
            self.lib.charming_fini()
            Runtime._active = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.fini()

    @property
    def n_pes(self) -> int:
        return self.info["n_pes"]

    def last_stats(self) -> RunStats:
        st = _lib.Stats()
        self.lib.charming_last_stats(C.byref(st))
        return RunStats(st.delivered, st.sent, st.stashed, st.revived, st.bytes_sent,
                        st.idle_polls, st.space_waits, st.kernel_ms, st.loop_ms, st.main_ms,
                        st.status, st.idle_ms, st.em_ms, st.deferred, st.ticket_ms, st.space_ms,
                        st.batched)

    # ---- built-in programs ---------------------------------------------------
    def hello(self) -> np.ndarray:
        n = 2 * self.n_pes
        out = (C.c_int * n)()
        nch = C.c_int(0)
        check(self.lib.charming_hello(out, n, C.byref(nch)), "charming_hello")
        return np.frombuffer(out, dtype=np.int32).copy()

    def refnum(self, reversed_order: bool = False) -> list[int]:
        out = (C.c_int * 2)()
        nd = C.c_int(0)
        fn = self.lib.charming_refnum_reversed if reversed_order else self.lib.charming_refnum
        check(fn(out, 2, C.byref(nd)), "charming_refnum")
        return [out[i] for i in range(nd.value)]

    def pingpong(self, sizes, round_trips: int, warmup: int = 10, seed: int = 1,
                 verify: bool = True):
        sizes = [int(s) for s in sizes]
        arr = (C.c_uint64 * len(sizes))(*sizes)
        res = (_lib.PingpongResult * len(sizes))()
        sm = (C.c_int * 2)()
        check(self.lib.charming_pingpong(arr, len(sizes), round_trips, warmup, seed,
                                         1 if verify else 0, res, sm), "charming_pingpong")
        rows = [dict(size=r.size, oneway_us=r.oneway_us, oneway_cycles=r.oneway_cycles,
                     checksum_errors=r.checksum_errors) for r in res]
        return rows, (sm[0], sm[1])

    def fanout(self, n_chares: int, msgs: int, payload: int, seed: int, mode: int):
        cap = n_chares * msgs
        log = np.zeros((cap, 8), dtype=np.uint32)
        n_logged = C.c_uint64(0)
        ms = C.c_double(0.0)
        check(self.lib.charming_fanout(n_chares, msgs, payload, seed, mode,
                                       log.ctypes.data_as(C.POINTER(C.c_uint32)), cap,
                                       C.byref(n_logged), C.byref(ms)), "charming_fanout")
        return log[: min(n_logged.value, cap)], ms.value

    def sm_pingpong(self, mode: int, round_trips: int = 10000):
        """SM-to-SM pingpong floor without the runtime (mode 0 flag, 1
        relaxed polls, 2 with block barriers, 3 the reference's slot
        scheme): one-way ns, cycles and the SM pair."""
        ns, cyc = C.c_double(0.0), C.c_double(0.0)
        sm = (C.c_int * 2)()
        check(self.lib.charming_sm_pingpong(mode, round_trips, C.byref(ns), C.byref(cyc), sm),
              "charming_sm_pingpong")
        return {"oneway_ns": ns.value, "oneway_cycles": cyc.value, "sm_pair": (sm[0], sm[1])}

    def sweep_bench(self, dtype: str, w: int, h: int, depth: int, passes: int, n_blocks: int = 0,
                    variant: int = 0) -> float:
        """Kernel ms of `passes` passes over n_blocks chare blocks of w x h
        (sweeps only, no messages); n_blocks 0: one per PE."""
        ms = C.c_double(0.0)
        check(self.lib.charming_sweep_bench(_lib.F64 if dtype == "f64" else _lib.F32, w, h, depth, passes,
                                            n_blocks or self.n_pes, variant, C.byref(ms)),
              "charming_sweep_bench")
        return ms.value

    def async_wait_chain(self, n_chares: int, broken: bool = False):
        """Wake order of a chain of async_waits; returns (status, order).
        A broken chain leaves the last chare waiting, so its run ends with
        an error status, which is returned rather than raised."""
        order = (C.c_int * n_chares)()
        rc = self.lib.charming_async_wait_chain(n_chares, 1 if broken else 0, order, n_chares)
        if rc and not broken:
            check(rc, "charming_async_wait_chain")
        return rc, [order[i] for i in range(n_chares)]

    def user_heap_check(self, n_chares: int, blocks: int, rounds: int, seed: int = 5):
        out = (C.c_uint64 * 7)()
        check(self.lib.charming_user_heap_check(n_chares, blocks, rounds, seed, out),
              "charming_user_heap_check")
        keys = ("taken", "bad", "failed", "checked", "freed", "done", "bytes")
        return {k: int(out[i]) for i, k in enumerate(keys)}

    def jacobi3d(self, grid: np.ndarray, sweeps: int):
        """`sweeps` 7-point FP64 sweeps of an (nz+2, ny+2, nx+2) grid; returns
        (result, device ms of the sweeps)."""
        g = np.ascontiguousarray(grid, dtype=np.float64).copy()
        nz, ny, nx = (d - 2 for d in g.shape)
        ms = C.c_double(0.0)
        check(self.lib.charming_jacobi3d(nx, ny, nz, sweeps, g.ctypes.data_as(C.POINTER(C.c_double)),
                                         C.byref(ms)), "charming_jacobi3d")
        return g, ms.value

    def decomp1d(self, n_chares: int, nx: int, ny: int, iters: int, mode: int):
        """jacobi2d-decomp1d: (ny-2) x nx float32 bands after `iters`
        iterations (mode 0 signals waited in the entry method, 1 async_wait,
        2 messages) and the loop's ms."""
        out = np.zeros((ny - 2, nx), dtype=np.float32)
        ms = C.c_double(0.0)
        check(self.lib.charming_jacobi2d_decomp1d(n_chares, nx, ny, iters, mode,
                                                  out.ctypes.data_as(C.POINTER(C.c_float)), C.byref(ms)),
              "charming_jacobi2d_decomp1d")
        return out, ms.value

    def jacobi1d(self, n_chares: int, width: int, sweeps: int):
        out = np.zeros(n_chares * width + 4, dtype=np.float64)
        ms = C.c_double(0.0)
        check(self.lib.charming_jacobi1d(n_chares, width, sweeps,
                                         out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(ms)),
              "charming_jacobi1d")
        return out, ms.value


def runtime(**overrides) -> Runtime:
    """The process-wide runtime, created on first use with `overrides`."""
    if Runtime._active is None:
        return Runtime(**overrides)
    return Runtime._active
