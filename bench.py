#!/usr/bin/env python3
"""Benchmark: Jacobi2d chares on one B200 (replicas on N GPUs).

Headline workload: jacobi2d 8192 x 8192 FP64, one chare per PE (148 on a
B200), halos exchanged as runtime messages, 100 sweeps per step (the
reference's default iteration count, examples/jacobi2d/jacobi2d.cu:12).
Metric: GLUP/s = interior points x sweeps / time.

The same JSON line carries the other workloads of the metric (skipped with
--headline-only):
  messaging  pingpong 8 B..1 MiB (10,000 round trips per size, payloads
             checksummed on the device) and fan-out 4096 chares x 16 x 64 B
             with refnums 0..15 (msgs/s)
  batched    64 uneven FP64 problems (sides log-uniform in [64, 2048]),
             500 sweeps, one launch replayed from a CUDA graph, launch
             configuration picked by the autotuner
  precision  the batched set plus one 8192^2 problem in FP32 with the FP64
             residual every 10 sweeps, stop at 1e-5 or 5000 sweeps; GLUP/s
             against the plain FP64 headline and the max-abs error against
             the FP64 grids after the same sweep counts
  serving    Poisson arrivals at 200 req/s of FP32 solves (sides log-uniform
             in [128, 4096], tol 1e-5, cap 5000 sweeps) into one running
             scheduler under a 120 GB HBM budget; p50/p99 latency, solves/s

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs under torchrun as independent replicas (the problem does not shard
across GPUs here); value is the sum over ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Jacobi2d GLUP/s + msgs/s on 1 B200, plain FP64 vs batched FP32; solve p99 ms"
UNIT = "GLUP/s"
NX = NY = 8192
SWEEPS = 100
BYTES_PER_LUP = 16  # FP64: one 8-byte read + one 8-byte write per point


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region:
    NVML read every 10 ms from a thread (read-only queries), or nvidia-smi
    every 200 ms when NVML is unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []  # (sm_mhz, max_mhz, set of reasons)
        self.proc = self.path = self.thread = None
        self.stop = False
        self.source = None

    def _nvml_sample(self, nv, h, mx):
        try:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            rs = {name for name, attr in self.REASONS if bits & getattr(nv, attr)}
            self.samples.append((float(sm), float(mx), rs))
        except Exception:
            pass

    def _nvml_loop(self, nv, h, mx):
        while not self.stop:
            self._nvml_sample(nv, h, mx)
            time.sleep(0.01)

    def __enter__(self):
        try:
            import threading

            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.device)
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._nvml = (nv, h, mx)
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h, mx), daemon=True)
            self.thread.start()
            self.source = "nvml 10 ms"
            return self
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi 200 ms"
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread:
            # one more reading at the end of the timed region (the sampling
            # thread may have had little time during a short region)
            self._nvml_sample(*self._nvml)
            self.stop = True
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            try:
                names = [n for n, _ in self.REASONS]
                for line in open(self.path):
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                        rs = {n for n, v in zip(names, parts[5:9]) if v.lower().startswith("active")}
                        self.samples.append((float(parts[1]), float(parts[2]), rs))
            except OSError:
                pass
            finally:
                os.unlink(self.path)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [x[0] for x in self.samples]
        loaded = [v for v in sm if v > 0.5 * max(sm)] or sm
        reasons = sorted(set().union(*(x[2] for x in self.samples)))
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": self.samples[0][1],
                "samples": len(self.samples), "source": self.source, "reasons": reasons}


def cpu_baseline(target_s: float = 12.0, threads: int | None = None) -> dict:
    """The same FP64 Jacobi arithmetic on the host cores (OpenMP, the
    oracle's port of the reference stencil), on a bounded sample of the
    workload: the 8192^2 grid for as many sweeps as fit in ~target_s
    (calibrated on a few sweeps first)."""
    from charming_b200.jacobi import initial_grid
    from oracle import jacobi as oj
    threads = threads or os.cpu_count() or 1
    os.environ.setdefault("OMP_PROC_BIND", "close")
    g = initial_grid(NX, NY, (1.0, 0.0, 0.0, 0.0))
    oj.jacobi2d(g, 2, threads=threads)  # thread pool and pages warm
    n, t1 = 8, 0.0
    while True:  # calibrate on runs of at least ~1 s
        t0 = time.perf_counter()
        oj.jacobi2d(g, n, threads=threads)
        dt0 = time.perf_counter() - t0
        t1 = dt0 / n
        if dt0 > 1.0 or n >= 4096:
            break
        n *= 4
    sweeps = int(max(4, min(20000, target_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    oj.jacobi2d(g, sweeps, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": NX * NY * sweeps / dt / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"jacobi2d {NX}x{NY} FP64, {sweeps} sweeps, OpenMP ({dt:.1f} s)"}


def choose_decomposition(n_pes: int, nx: int, ny: int) -> tuple[int, int]:
    """One chare per PE; px (columns of chares) small so block rows are long
    (each block row streams through the bulk-copy pipeline)."""
    best = None
    for px in range(1, n_pes + 1):
        if n_pes % px:
            continue
        py = n_pes // px
        w = nx / px
        if w > 2048 or px > nx or py > ny:
            continue
        score = (nx / px + ny / py)  # halo surface per chare
        if w < 1024:
            score *= 1.5
        if best is None or score < best[0]:
            best = (score, px, py)
    return (best[1], best[2]) if best else (1, n_pes)


def set_workload(n: int, sweeps: int) -> None:
    global NX, NY, SWEEPS
    NX = NY = n
    SWEEPS = sweeps


def dist_setup(backend: str | None = None):
    """Replica ranks from the torchrun environment: NCCL on GPUs, gloo
    without one (the CPU tests of this plumbing)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1:
        return None, rank, local, world
    import datetime

    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist, rank, local, world


def _on_gpu(dist) -> bool:
    return dist.get_backend() == "nccl"


def dist_max(dist, x: float, local: int) -> float:
    """Max over ranks (the job's time is its slowest rank's)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}" if _on_gpu(dist) else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, local: int) -> None:
    if dist is not None:
        import torch
        if _on_gpu(dist):
            dist.barrier(device_ids=[local])
            torch.cuda.synchronize(local)
        else:
            dist.barrier()


def replica_value(lups_per_rank_step: float, steps: int, world: int, max_ms: float) -> float:
    """Whole-job GLUP/s of N replicas: all ranks' updates over the slowest
    rank's time."""
    return lups_per_rank_step * steps * world / (max_ms * 1e-3) / 1e9


def traffic_from_profiles(workload: str):
    """Per-launch DRAM bytes of the scheduler kernel from the committed ncu
    summary (profiles/ncu_traffic.json), scaled to this workload's size."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            d = json.load(f)
        e = d.get(workload)
        return e["bytes_per_launch"] if e else None
    except (OSError, ValueError, KeyError):
        return None


def run_reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    samples = []
    per_step_s = 4.0
    for _ in range(args.warmup):
        cpu_baseline(target_s=1.0, threads=threads)
    for _ in range(args.steps):
        samples.append(cpu_baseline(target_s=per_step_s, threads=threads))
    v = statistics.mean(s["value"] for s in samples)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": NX * NY * SWEEPS / (v * 1e9) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(args, None),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": samples[-1]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def messaging_suite(seed: int = 0xC2) -> dict:
    """C2a pingpong and C2b fan-out. Message rate scales with PEs per SM
    (each PE handles one message at a time with its whole block), so the
    fan-out runs on four 128-thread PEs per SM (the default configuration's
    rate is reported beside it). Pingpong runs on the default 512-thread
    PEs, whose payload copies are the fastest; one 128-thread PE per SM
    answers small messages sooner, reported beside it."""
    from charming_b200.runtime import Runtime
    n = 4096 * 16
    rt = Runtime()
    _, ms_def = rt.fanout(4096, 16, 64, seed, 1)
    _, ms_def_fifo = rt.fanout(4096, 16, 64, seed, 0)
    sizes = [1 << k for k in range(3, 21)]
    rows, sm = rt.pingpong(sizes, 10000, warmup=200, seed=seed, verify=True)
    st = rt.last_stats()
    rt = Runtime(pes_per_sm=1, threads_per_pe=128)
    small, _ = rt.pingpong([8, 64, 1024], 10000, warmup=200, seed=seed, verify=True)
    floors = {name: rt.sm_pingpong(mode, 10000) for mode, name in
              ((0, "flag_release_acquire"), (1, "flag_relaxed_poll_fence"), (2, "flag_with_block_barriers"),
               (3, "reference_slot_scheme"))}
    rt = Runtime(pes_per_sm=4, threads_per_pe=128)
    log, ms = rt.fanout(4096, 16, 64, seed, 1)
    fst = rt.last_stats()
    _, ms_fifo = rt.fanout(4096, 16, 64, seed, 0)
    Runtime()
    return {
        "pingpong": {"runtime": "1 PE of 512 threads per SM", "sm_pair": list(sm), "round_trips": 10000,
                     "oneway_ns_128_thread_pe": {str(r["size"]): round(r["oneway_us"] * 1e3, 1) for r in small},
                     "oneway_ns": {str(r["size"]): round(r["oneway_us"] * 1e3, 1) for r in rows},
                     "oneway_cycles": {str(r["size"]): round(r["oneway_cycles"], 1) for r in rows},
                     "checksum_errors": int(sum(r["checksum_errors"] for r in rows)),
                     "status": st.status,
                     "floor": {k: {"oneway_ns": round(v["oneway_ns"], 1), "oneway_cycles": round(v["oneway_cycles"], 1)}
                               for k, v in floors.items()},
                     "floor_note": "two thread blocks on different SMs bouncing a counter without the runtime "
                                   "(charming_sm_pingpong); reference_slot_scheme restates examples/baseline"},
        "fanout": {"runtime": "4 PEs of 128 threads per SM", "chares": 4096, "msgs_per_chare": 16,
                   "payload_bytes": 64, "refnums": "0..15",
                   "ms": ms, "msgs_per_s": n / (ms * 1e-3), "delivered": int(len(log)),
                   "stashed": fst.stashed, "status": fst.status,
                   "fifo_msgs_per_s": n / (ms_fifo * 1e-3),
                   "default_runtime_msgs_per_s": n / (ms_def * 1e-3),
                   "default_runtime_fifo_msgs_per_s": n / (ms_def_fifo * 1e-3),
                   "checked": "counts, per-pair FIFO and checksums against the CPU model in tests"},
        "cpu_baseline": messaging_cpu_baseline(seed),
    }


def messaging_cpu_baseline(seed: int) -> dict:
    """The same fan-out (FIFO mode) and pingpong on the host's cores, one
    MPSC inbox per thread (oracle/msg_cpu.c)."""
    from oracle import msg_cpu
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_PROC_BIND", "close")
    reps = [msg_cpu.fanout(4096, 16, 64, seed, threads)[0] for _ in range(21)]
    pp = {str(b): round(msg_cpu.pingpong_oneway_s(b, 10000 if b < (1 << 20) else 1000, seed) * 1e9, 1)
          for b in (8, 4096, 65536, 1 << 20)}
    return {"kind": "port", "cores": threads,
            "fanout_fifo_msgs_per_s": 4096 * 16 / statistics.median(reps),
            "pingpong_oneway_ns": pp,
            "sample": "fan-out 4096 x 16 x 64 B (FIFO), median of 21; pingpong 10,000 round trips "
                      "(1,000 for 1 MiB) between two threads"}


def _omp_threads() -> int:
    os.environ.setdefault("OMP_PROC_BIND", "close")
    return os.cpu_count() or 1


def _sweep_inplace(g: np.ndarray, sweeps: int, threads: int) -> None:
    """OpenMP oracle sweeps on the grid in place (FP64 or FP32)."""
    import ctypes as C

    from oracle import jacobi as oj
    ny, nx = g.shape[0] - 2, g.shape[1] - 2
    if g.dtype == np.float64:
        oj.lib().oracle_jacobi2d_f64_omp(g.ctypes.data_as(C.POINTER(C.c_double)), nx, ny, sweeps, threads)
    else:
        oj.lib().oracle_jacobi2d_f32(g.ctypes.data_as(C.POINTER(C.c_float)), nx, ny, sweeps, threads)


def cpu_set_baseline(probs, dtype: str, target_s: float = 10.0) -> dict:
    """The batched (or precision) problem set on the host cores: every problem
    swept by the OpenMP oracle (FP64, or FP32 with the FP64 residual every
    10 sweeps for the precision set), for a sweep count per problem scaled so
    the whole sample takes about target_s; GLUP/s over the sample."""
    from charming_b200.jacobi import initial_grid
    from oracle import jacobi as oj
    threads = _omp_threads()
    npdt = np.float64 if dtype == "f64" else np.float32
    grids = [np.ascontiguousarray(initial_grid(p.nx, p.ny, p.bc, npdt)) for p in probs]
    points = sum(p.nx * p.ny for p in probs)

    def run(sweeps: int) -> float:
        t0 = time.perf_counter()
        for p, g in zip(probs, grids):
            if dtype == "f64":
                _sweep_inplace(g, sweeps, threads)
            else:
                done = 0
                while done < sweeps:
                    k = min(10, sweeps - done)
                    _sweep_inplace(g, k, threads)
                    oj.residual(g)
                    done += k
        return time.perf_counter() - t0
    t1 = run(10) / 10
    sweeps = int(max(10, min(5000, target_s / max(t1, 1e-9))))
    sweeps = sweeps // 10 * 10
    dt = run(sweeps)
    return {"value": points * sweeps / dt / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"all {len(probs)} problems, {sweeps} sweeps each ({dtype}"
                      f"{', FP64 residual every 10 sweeps' if dtype == 'f32' else ''}; {dt:.1f} s)"}


def cpu_serving_baseline(probs, arrive, sweeps, target_s: float = 12.0) -> dict:
    """The serving trace on the host cores, from a bounded sample: the
    OpenMP FP32 sweep (FP64 residual every 10 sweeps, as the server checks)
    is timed on grids of the trace's smallest, middle and largest sides for
    about target_s in all; each request's solve time is then its points x
    the sweeps the GPU ran for it x the time per update measured at the
    nearest size (log-interpolated), and the requests are served one after
    another, each on all cores, from their arrival times (a FIFO queue on the
    same arrivals). Solving all 20,000 requests on the host would take
    hours: one 4096^2 request alone takes over a minute."""
    from charming_b200.jacobi import initial_grid
    from oracle import jacobi as oj
    threads = _omp_threads()
    sides = sorted({int(p.nx) for p in probs})
    pick = sorted({sides[0], sides[len(sides) // 2], sides[-1]})
    per_lup = {}
    t_all = time.perf_counter()
    for side in pick:
        g = np.ascontiguousarray(initial_grid(side, side, (1.0, 0.5, 0.25, 0.0), np.float32))
        t0 = time.perf_counter()
        _sweep_inplace(g, 10, threads)
        oj.residual(g)
        t10 = time.perf_counter() - t0
        n = max(10, int(target_s / len(pick) / max(t10 / 10, 1e-9)) // 10 * 10)
        t0 = time.perf_counter()
        for _ in range(n // 10):
            _sweep_inplace(g, 10, threads)
            oj.residual(g)
        per_lup[side] = (time.perf_counter() - t0) / (side * side * n)
    xs = np.log([float(s * s) for s in pick])
    ys = np.array([per_lup[s] for s in pick])
    busy, lat, lups = 0.0, [], 0
    for p, at, sw in zip(probs, arrive, sweeps):
        pts = p.nx * p.ny
        t = pts * sw * float(np.interp(np.log(float(pts)), xs, ys))
        busy = max(busy, at) + t
        lat.append(busy - at)
        lups += pts * sw
    span = busy - arrive[0]
    return {"kind": "port", "cores": threads, "requests": len(probs), "solves_per_s": len(probs) / span,
            "p50_ms": float(np.percentile(lat, 50)) * 1e3, "p99_ms": float(np.percentile(lat, 99)) * 1e3,
            "served_glups": lups / span / 1e9,
            "ns_per_update": {str(s): round(per_lup[s] * 1e9, 3) for s in pick},
            "sample": f"FP32 sweeps + FP64 residual timed on {pick} grids ({time.perf_counter() - t_all:.1f} s); "
                      "each request's solve time = points x the GPU's sweep count x the measured time per update "
                      "(log-interpolated by size); requests served one at a time on all cores, FIFO from their "
                      "arrival times"}


def batched_suite(steps: int = 3, warmup: int = 3) -> dict:
    """C3: the 64-problem uneven FP64 set, 500 sweeps, CUDA graph, autotuned."""
    from charming_b200.batch import autotune, uneven_set
    from charming_b200.jacobi import Jacobi2D
    probs = uneven_set(max_sweeps=500)
    tune = autotune(probs, "f64")
    best = tune.best
    points = sum(p.nx * p.ny for p in probs)
    with Jacobi2D(probs, dtype="f64", chare_side=best.chare_side, use_graph=True) as j:
        for _ in range(warmup):
            j.run()
        ts = [j.run() for _ in range(steps)]
        info = j.info()
    ms = statistics.mean(ts)
    # the same set with chare sides outside the config's 64/128/256 choice
    from charming_b200.batch import Candidate
    ext = autotune(probs, "f64", candidates=[Candidate(sd, pe, 4 << 20) for sd in (512, 1024)
                                             for pe in (1, 2, 4)])
    return {"outside_config": {"chare_sides": [512, 1024], "glups": ext.best.glups,
                               "autotune": ext.as_dict()},
            "workload": "64 square FP64 problems, sides log-uniform in [64, 2048] (seed 0xC3), "
                        "500 sweeps, one launch from a CUDA graph",
            "glups": points * 500 / (ms * 1e-3) / 1e9, "ms_per_launch": ms, "launches": steps,
            "points": points, "chares": info["n_chares"], "autotune": tune.as_dict(),
            "cpu_baseline": cpu_set_baseline(probs, "f64")}


def precision_suite(plain_fp64_glups: float, steps: int = 2, warmup: int = 1) -> dict:
    """C4: the batched set plus 8192^2 in FP32 sweeps with the FP64 residual
    (every 10 sweeps, stop at 1e-5 or 5000 sweeps); max-abs error against
    FP64 grids after the same sweep counts (the FP64 path equals the serial
    oracle bit for bit)."""
    from charming_b200.batch import _uniform, autotune, default_candidates, uneven_set
    from charming_b200.jacobi import Jacobi2D, Problem
    bc = tuple(_uniform(0xC4, k) for k in range(4))
    probs = uneven_set(max_sweeps=5000, check_every=10, tol=1e-5)
    # the single 8192^2 problem is cut like the plain FP64 headline problem
    # (one chare per PE of one 512-thread PE per SM); the config's 64/128/256
    # chare blocks are the batched set's
    from charming_b200.runtime import Runtime as _Rt
    bpx, bpy = choose_decomposition(_Rt().n_pes, 8192, 8192)
    probs.append(Problem(8192, 8192, 5000, px=bpx, py=bpy, check_every=10, tol=1e-5, bc=bc))
    proxy = [Problem(p.nx, p.ny, 100, px=p.px, py=p.py, check_every=10, tol=0.0, bc=p.bc) for p in probs]
    cands = [c for c in default_candidates() if c.chare_side >= 128 and c.ring_bytes == (4 << 20)]
    tune = autotune(proxy, "f32", candidates=cands)
    side = tune.best.chare_side
    with Jacobi2D(probs, dtype="f32", chare_side=side, use_graph=True) as j:
        ts = []
        for k in range(warmup + steps):
            j.init()  # every launch solves from the initial state (outside the timed launch)
            t = j.run()
            if k >= warmup:
                ts.append(t)
        res = [j.result(i) for i in range(len(probs))]
        g32 = [j.store(i) for i in range(len(probs))]
    ms = statistics.mean(ts)
    lups = sum(p.nx * p.ny * r.sweeps for p, r in zip(probs, res))
    ref = [Problem(p.nx, p.ny, r.sweeps, bc=p.bc) for p, r in zip(probs, res)]
    err = 0.0
    with Jacobi2D(ref, dtype="f64", chare_side=side) as j64:
        j64.run()
        for i in range(len(ref)):
            g64 = j64.store(i)
            err = max(err, float(np.max(np.abs(g32[i].astype(np.float64) - g64))))
    glups = lups / (ms * 1e-3) / 1e9
    sw = [r.sweeps for r in res]
    # the same FP32 run with chare sides outside the config's 64/128/256 choice
    from charming_b200.batch import Candidate
    ext = autotune(proxy, "f32", candidates=[Candidate(sd, pe, 4 << 20) for sd in (512, 1024, 2048)
                                             for pe in (1, 2)])
    with Jacobi2D(probs, dtype="f32", chare_side=ext.best.chare_side, use_graph=True) as j:
        j.init()
        j.run()
        j.init()
        ms_ext = j.run()
        lups_ext = sum(p.nx * p.ny * j.result(i).sweeps for i, p in enumerate(probs))
    glups_ext = lups_ext / (ms_ext * 1e-3) / 1e9
    return {"workload": "the batched set with 5000-sweep caps plus one 8192^2 problem, FP32 "
                        "sweeps and storage, FP64 residual every 10 sweeps, tol 1e-5",
            "decomposition_8192": f"{bpx} x {bpy} chares, as the plain FP64 headline problem",
            "glups": glups, "ms_per_launch": ms, "launches": steps,
            "vs_plain_fp64": glups / plain_fp64_glups if plain_fp64_glups else None,
            "outside_config": {"chare_sides": [512, 1024, 2048], "glups": glups_ext,
                               "vs_plain_fp64": glups_ext / plain_fp64_glups if plain_fp64_glups else None,
                               "autotune": ext.as_dict()},
            "target_vs_plain_fp64": 1.8, "max_abs_err_vs_fp64": err, "target_max_abs_err": 1e-5,
            "sweeps_min": min(sw), "sweeps_max": max(sw),
            "stopped_by_tol": sum(1 for p, r in zip(probs, res) if r.sweeps < p.max_sweeps),
            "res_rel_8192": res[-1].res_last / res[-1].res0 if res[-1].res0 else None,
            "reference": "FP64 grids from the FP64 path (bit-identical to the serial oracle) "
                         "after each problem's FP32 sweep count",
            "autotune": tune.as_dict(),
            "cpu_baseline": cpu_set_baseline(probs, "f32")}


def serving_suite(n_req: int, rate: float = 200.0, seed: int = 0xC5, pes_per_sm: int = 1,
                  chare_side: int = 2048, max_inflight: int = 64, with_cpu: bool = True) -> dict:
    """C5: Poisson arrivals of FP32 solves into one running scheduler. The
    defaults are the fastest measured (600 requests, served GLUP/s): chares
    of 2048^2 on one 512-thread PE per SM 759; 1536^2 701; 1024^2 with 2 PEs
    per SM 655; 512^2 with 2 PEs per SM 512; 4096^2 (one chare per request)
    337."""
    import torch
    from charming_b200.batch import _uniform
    from charming_b200.jacobi import Problem
    from charming_b200.runtime import Runtime
    from charming_b200.serve import Server
    # several PEs per SM: the messages of one overlap the sweeps of another
    Runtime(pes_per_sm=pes_per_sm, threads_per_pe=512 // pes_per_sm)
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(np.log(128), np.log(4096), n_req)).round().astype(int)
    gaps = rng.exponential(1.0 / rate, n_req)
    arrive = np.cumsum(gaps) - gaps[0]
    probs = [Problem(int(s), int(s), 5000, check_every=10, tol=1e-5,
                     bc=tuple(float(v) for v in rng.uniform(0, 1, 4))) for s in sides]
    out = torch.empty((4098 * 4098,), dtype=torch.float32, pin_memory=True).numpy()
    budget = 120 * 10**9
    lat, service, lups_done = [], [], 0
    sweeps_of = [0] * n_req
    with Server(budget, max_inflight=max_inflight, workers_per_pe=16 // pes_per_sm, chare_side=chare_side,
                dtype="f32", deadline_s=600) as srv:
        t0 = time.monotonic()
        nxt = 0
        done = 0
        while done < n_req:
            now = time.monotonic() - t0
            while nxt < n_req and arrive[nxt] <= now:
                srv.submit(probs[nxt], nxt)
                nxt += 1
            for c in srv.poll():
                p = probs[c.tag]
                srv.fetch(c.tag, out[: (p.ny + 2) * (p.nx + 2)].reshape(p.ny + 2, p.nx + 2))
                srv.release(c.tag)
                lat.append(c.done_s - c.submit_s)
                service.append(c.done_s - c.admit_s)
                lups_done += p.nx * p.ny * c.sweeps
                sweeps_of[c.tag] = c.sweeps
                done += 1
            if time.monotonic() - t0 > 900:
                break
            time.sleep(0.0001)
        wall = time.monotonic() - t0
        stats = srv.stop()
    offered = sum(p.nx * p.ny * p.max_sweeps for p in probs) / max(arrive[-1], 1e-9)
    return {"workload": f"{n_req} FP32 solve requests, Poisson {rate:.0f} req/s, sides log-uniform "
                        "in [128, 4096], tol 1e-5 with the FP64 residual every 10 sweeps, cap 5000 "
                        f"sweeps, 120 GB HBM budget, chares of {chare_side}^2 on {pes_per_sm} PEs "
                        "per SM, each result fetched to the host",
            "requests": n_req, "completed": done, "wall_s": wall,
            "solves_per_s": done / wall, "p50_ms": float(np.percentile(lat, 50)) * 1e3,
            "p99_ms": float(np.percentile(lat, 99)) * 1e3,
            "service_p50_ms": float(np.percentile(service, 50)) * 1e3,
            "service_p99_ms": float(np.percentile(service, 99)) * 1e3,
            "offered_glups": offered / 1e9, "served_glups": lups_done / wall / 1e9,
            "peak_inflight": stats.get("peak_inflight"), "peak_bytes": stats.get("peak_bytes"),
            "cpu_baseline": cpu_serving_baseline(probs, arrive, sweeps_of) if with_cpu else None}


MULTI_GPU_CHILD = """
import json
from charming_b200.runtime import Runtime
out = {}
for v in (2, 1):
    rt = Runtime(virtual_devs=v)
    rows, _ = rt.pingpong([8, 64, 4096], round_trips=10000, warmup=100, seed=1, verify=False)
    seed = 0xC0FFEE + 4096 + 1
    rt.fanout(4096, 16, 64, seed, 1)
    log, ms = rt.fanout(4096, 16, 64, seed, 1)
    out[v] = {"pingpong_oneway_ns": {str(r["size"]): round(r["oneway_us"] * 1e3, 1) for r in rows},
              "fanout_msgs_per_s": 4096 * 16 / (ms * 1e-3), "n_pes": rt.n_pes}
    rt.fini()
print(json.dumps(out))
"""


def multi_gpu_suite() -> dict:
    """The multi-GPU transport (its own build of the library, so in a child
    process) on one B200: the 148 PEs form 2 virtual GPUs, each with its own
    inbox memory; PE 0 and PE 74 (pingpong) sit on different ones, and the
    fan-out's messages cross between them with system-scope tickets and
    flags. Beside it, the same build with one GPU."""
    r = subprocess.run([sys.executable, "-c", MULTI_GPU_CHILD], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    if r.returncode != 0:
        return {"error": r.stderr[-500:]}
    res = json.loads(r.stdout.strip().splitlines()[-1])
    two, one = res["2"], res["1"]
    return {"build": "libcharming_b200_multi.so", "virtual_gpus": 2,
            "pingpong_oneway_ns_cross_gpu": two["pingpong_oneway_ns"],
            "fanout_msgs_per_s_2_gpus": two["fanout_msgs_per_s"],
            "one_gpu_same_build": {"pingpong_oneway_ns": one["pingpong_oneway_ns"],
                                   "fanout_msgs_per_s": one["fanout_msgs_per_s"]},
            "workload": "pingpong 8/64/4096 B, 10000 round trips; fan-out 4096 chares x 16 msgs of 64 B, "
                        "refnums 0..15, 1 PE of 512 threads per SM",
            "note": "virtual GPUs: a peer's rings are this GPU's memory, so NVLink's latency is not in "
                    "these numbers; the difference to one GPU is the system-scope protocol"}


def run_suites(args, headline_glups: float) -> dict:
    out = {}
    for name, fn in (("messaging", lambda: messaging_suite()),
                     ("multi_gpu", lambda: multi_gpu_suite()),
                     ("batched", lambda: batched_suite()),
                     ("precision", lambda: precision_suite(headline_glups)),
                     ("serving", lambda: serving_suite(args.serve_requests))):
        if name in args.skip:
            continue
        t0 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as e:  # report, keep the line
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["suite_s"] = round(time.perf_counter() - t0, 1)
    return out


def exchange_depth(args) -> int:
    """Sweeps per halo exchange the run uses (the library's choice for 0:
    6 without residual checks)."""
    if args.pipeline:
        return 1
    return min(args.depth if args.depth > 0 else 6, 8)


def workload_config(args, decomp) -> dict:
    px, py = decomp if decomp else (args.px, args.py)
    dep = exchange_depth(args)
    return {"workload": f"jacobi2d {NX}x{NY} FP64, {SWEEPS} sweeps per step, halos as messages"
                        + (f" every {dep} sweeps" if dep > 1 else ""),
            "grid": [NX, NY], "sweeps_per_step": SWEEPS, "chares": [px, py],
            "sweeps_per_exchange": dep,
            "parallelism": f"replicas x{args.gpus}", "l2": "inputs larger than L2 (1.07 GB/sweep)"}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="charming", choices=["charming", "reference"])
    ap.add_argument("--px", type=int, default=0)
    ap.add_argument("--py", type=int, default=0)
    ap.add_argument("--pipeline", type=int, default=0, help="1: TMA row pipeline, 0: direct loads")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--nx", type=int, default=NX, help="grid size (profiling runs)")
    ap.add_argument("--sweeps", type=int, default=SWEEPS)
    ap.add_argument("--tile-w", type=int, default=0)
    ap.add_argument("--depth", type=int, default=0,
                    help="sweeps per halo exchange (ghost depth), 0: 6 (direct) / 1 (TMA)")
    ap.add_argument("--threads-per-pe", type=int, default=512)
    ap.add_argument("--pes-per-sm", type=int, default=1)
    ap.add_argument("--small-buffers", action="store_true",
                    help="1 MiB inbox rings and stashes (smaller device footprint for ncu)")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the messaging, batched, precision and serving workloads")
    ap.add_argument("--skip", default="", help="comma-separated workloads to skip")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests of the serving workload (the full stream is 20000)")
    args = ap.parse_args()
    set_workload(args.nx, args.sweeps)

    dist, rank, local, world = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, rank)
        if dist is not None:
            dist.destroy_process_group()
        return 0

    from charming_b200 import runtime
    from charming_b200.jacobi import Jacobi2D, Problem, initial_grid
    cfg = dict(device=local, threads_per_pe=args.threads_per_pe, pes_per_sm=args.pes_per_sm)
    if args.small_buffers:
        cfg.update(ring_bytes=1 << 20, stash_bytes=2 << 20, max_msg_bytes=(256 << 10))
    rt = runtime(**cfg)
    n_pes = rt.n_pes
    px, py = (args.px, args.py) if args.px and args.py else choose_decomposition(n_pes, NX, NY)
    prob = Problem(NX, NY, SWEEPS, px=px, py=py, bc=(1.0, 0.0, 0.0, 0.0))
    j = Jacobi2D([prob], dtype="f64", pipeline=bool(args.pipeline), balance=True,
                 tile_w=args.tile_w, depth=args.depth)
    lib = rt.lib
    import ctypes as C

    for _ in range(max(3, args.warmup)):
        j.run()
    barrier(dist, local)
    # the K steps go to the device back to back, synchronised once: the
    # host's work between runs (status and statistics reads, the Python
    # loop) is not part of the job's throughput, and on a busy host it
    # varied from 0.1 to 2.8 ms per step
    with ClockSampler(local) as clk:
        lib.charming_timer_start()
        runs_ms = j.run_n(args.steps)
        ms = C.c_double(0.0)
        lib.charming_timer_stop(C.byref(ms))
    launch_ms = [runs_ms / args.steps]
    barrier(dist, local)
    total_ms = dist_max(dist, ms.value, local)
    clocks = clk.summary()
    stats = rt.last_stats()
    lups = NX * NY * SWEEPS
    value = replica_value(lups, args.steps, world, total_ms)
    info = j.info()
    msgs_per_s = info["halo_msgs_per_sweep"] * SWEEPS * args.steps / (total_ms * 1e-3)

    # e2e: every step copies its input grid in from pinned host memory,
    # solves it and copies the result grid out, through the public
    # streaming call (charming_jacobi2d_solve_stream): the copies of step
    # k+1's input and step k-1's result overlap step k's solve
    e2e = None
    if not args.no_e2e:
        import torch
        g0 = initial_grid(NX, NY, prob.bc)
        h_in = torch.empty(g0.shape, dtype=torch.float64, pin_memory=True).numpy()
        h_out = torch.empty(g0.shape, dtype=torch.float64, pin_memory=True).numpy()
        h_in[...] = g0
        j.solve_stream(0, [h_in] * 2, [h_out] * 2)
        barrier(dist, local)
        e2e_ms = j.solve_stream(0, [h_in] * args.steps, [h_out] * args.steps)
        barrier(dist, local)
        e2e_ms = dist_max(dist, e2e_ms, local)
        nbytes = h_in.nbytes
        e2e = {"value": lups * args.steps * world / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "ms_per_step": e2e_ms / args.steps,
               "api": "charming_jacobi2d_solve_stream (copies of neighbouring steps overlap each solve)"}

    peaks = measured_peaks()
    peak = peaks.get("hbm_gbs")
    mean_launch = statistics.mean(launch_ms)
    achieved = BYTES_PER_LUP * lups / (mean_launch * 1e-3) / 1e9
    dep = exchange_depth(args)
    workload = f"jacobi2d_{NX}x{NY}_f64_{px}x{py}_d{dep}"
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak if peak else 6650.0,
            "unit": "GB/s", "frac": achieved / (peak if peak else 6650.0),
            "traffic": traffic_from_profiles(workload),
            "peak_source": "measured" if peak else "fallback",
            "kernel": "charming_scheduler_kernel (persistent; sweeps + halo messages)",
            "algorithmic_bytes_per_launch": BYTES_PER_LUP * lups,
            "traffic_key": workload}
    if dep > 1:
        roof["effective"] = (f"achieved counts 16 B per lattice update per sweep; a pass of {dep} "
                             "sweeps reads and writes each block once, so DRAM moves about "
                             f"1/{dep} of that and frac can exceed 1 (effective bandwidth)")
    j.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
    suites = {}
    if rank == 0 and world == 1 and not args.headline_only:
        args.skip = [x for x in args.skip.split(",") if x]
        suites = run_suites(args, value)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, (px, py)),
            "msgs_per_s": msgs_per_s, "halo_msgs_per_sweep": info["halo_msgs_per_sweep"],
            "last_launch": {"ms": info["last_run_ms"], "sweep_ms_max_pe": info["sweep_ms_max"],
                            "sweep_ms_mean_pe": info["sweep_ms_mean"],
                            "send_ms_mean_pe": info["send_ms_mean"],
                            "halo_em_ms_mean_pe": info["halo_ms_mean"], "main_ms": stats.main_ms,
                            "em_ms_mean_pe": stats.em_ms, "idle_ms_mean_pe": stats.idle_ms,
                            "loop_ms": stats.loop_ms, "stashed": stats.stashed,
                            "delivered": stats.delivered},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            # per timed step: the reset kernel, the scheduler kernel and the
            # status latch of charming_jacobi2d_run_n
            "gpu_launches": 3 * args.steps, "status": stats.status,
            "runtime": {k: rt.info[k] for k in ("n_pes", "threads_per_pe", "smem_bytes_per_pe",
                                                "smem_scratch_bytes", "regs_per_thread")},
        }
        line.update(suites)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
