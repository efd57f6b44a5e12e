#!/usr/bin/env python3
"""Benchmark: Jacobi2d chares on one B200 (replicas on N GPUs).

Headline workload: jacobi2d 8192 x 8192 FP64, one chare per PE (148 on a
B200), halos exchanged as runtime messages every sweep, 100 sweeps per step
(the reference's default iteration count, examples/jacobi2d/jacobi2d.cu:12).
Metric: GLUP/s = interior points x sweeps / time.

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
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": sorted(reasons)}


def cpu_baseline(target_s: float = 10.0, threads: int | None = None) -> dict:
    """The same FP64 Jacobi arithmetic on the host cores (OpenMP, the
    oracle's port of the reference stencil), on a bounded sample of the
    workload: the 8192^2 grid for as many sweeps as fit in ~target_s."""
    from charming_b200.jacobi import initial_grid
    from oracle import jacobi as oj
    threads = threads or os.cpu_count() or 1
    os.environ.setdefault("OMP_PROC_BIND", "close")
    g = initial_grid(NX, NY, (1.0, 0.0, 0.0, 0.0))
    t0 = time.perf_counter()
    oj.jacobi2d(g, 1, threads=threads)
    t1 = time.perf_counter() - t0
    sweeps = int(max(2, min(200, target_s / max(t1, 1e-6))))
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


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1:
        return None, rank, local, world
    import datetime

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist, rank, local, world


def dist_max(dist, x: float, local: int) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, local: int) -> None:
    if dist is not None:
        import torch
        dist.barrier(device_ids=[local])
        torch.cuda.synchronize(local)


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
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(args, None),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": samples[-1]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def exchange_depth(args) -> int:
    """Sweeps per halo exchange the run uses (the library's choice for 0)."""
    if args.pipeline:
        return 1
    return min(args.depth if args.depth > 0 else 4, 4)


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
                    help="sweeps per halo exchange (ghost depth), 0: 4 (direct) / 1 (TMA)")
    ap.add_argument("--small-buffers", action="store_true",
                    help="1 MiB inbox rings and stashes (smaller device footprint for ncu)")
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
    cfg = dict(device=local)
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
    launch_ms = []
    with ClockSampler(local) as clk:
        lib.charming_timer_start()
        for _ in range(args.steps):
            launch_ms.append(j.run())
        ms = C.c_double(0.0)
        lib.charming_timer_stop(C.byref(ms))
    barrier(dist, local)
    total_ms = dist_max(dist, ms.value, local)
    clocks = clk.summary()
    stats = rt.last_stats()
    lups = NX * NY * SWEEPS
    value = lups * args.steps * world / (total_ms * 1e-3) / 1e9
    info = j.info()
    msgs_per_s = info["halo_msgs_per_sweep"] * SWEEPS * args.steps / (total_ms * 1e-3)

    # e2e: host grid in (pinned), solve, host grid out, every step
    e2e = None
    if not args.no_e2e:
        import torch
        g0 = initial_grid(NX, NY, prob.bc)
        h_in = torch.empty(g0.shape, dtype=torch.float64, pin_memory=True).numpy()
        h_out = torch.empty(g0.shape, dtype=torch.float64, pin_memory=True).numpy()
        h_in[...] = g0
        j.load(0, h_in)
        j.run()
        j.store(0, h_out)
        barrier(dist, local)
        lib.charming_timer_start()
        for _ in range(args.steps):
            j.load(0, h_in)
            j.run()
            j.store(0, h_out)
        ms2 = C.c_double(0.0)
        lib.charming_timer_stop(C.byref(ms2))
        barrier(dist, local)
        e2e_ms = dist_max(dist, ms2.value, local)
        nbytes = h_in.nbytes
        e2e = {"value": lups * args.steps * world / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "ms_per_step": e2e_ms / args.steps}

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
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
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
                            "loop_ms": stats.loop_ms, "stashed": stats.stashed,
                            "delivered": stats.delivered},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": 2 * args.steps, "status": stats.status,
            "runtime": {k: rt.info[k] for k in ("n_pes", "threads_per_pe", "smem_bytes_per_pe",
                                                "smem_scratch_bytes", "regs_per_thread")},
        }
        print(json.dumps(line), flush=True)
    j.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
