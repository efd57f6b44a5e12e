"""Batched uneven Jacobi2d problems in one persistent launch, and the
autotuner that picks the launch configuration for a problem set.

A batch is any list of problems; ``uneven_set`` draws the seeded set of
square Dirichlet problems with log-uniform sides (64 problems of side
64..2048, each boundary edge uniform in [0, 1], interiors 0). The whole set
runs in one scheduler launch replayed from a captured CUDA graph
(``Jacobi2D(use_graph=True)``).

``autotune`` times the set under each candidate configuration -- chare
block side (64, 128, 256), PEs per SM (1 block of 512 threads, 2 of 256 or
4 of 128) and inbox ring depth -- and returns the fastest. Every candidate computes
bit-identical results (the decomposition only changes where a point is
updated, not its arithmetic), so the choice is free to follow speed alone.
"""
from __future__ import annotations

import itertools
import json
import os
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import CharmingError
from .jacobi import Jacobi2D, Problem
from .runtime import Runtime

MASK64 = (1 << 64) - 1


def _mix64(z: int) -> int:
    """SplitMix64 finaliser (the generator the seeded workloads use)."""
    z = (z + 0x9E3779B97F4A7C15) & MASK64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def _uniform(seed: int, i: int) -> float:
    return (_mix64((seed * 0x100000001B3 + i) & MASK64) >> 11) * (1.0 / (1 << 53))


def uneven_set(seed: int = 0xC3, n: int = 64, lo: int = 64, hi: int = 2048, max_sweeps: int = 500,
               check_every: int = 0, tol: float = 0.0) -> list[Problem]:
    """n square problems, side = round(exp(U(log lo, log hi))) by seed, each
    boundary edge U(0, 1) by seed, interior 0."""
    out = []
    for p in range(n):
        u = _uniform(seed, 5 * p)
        side = int(round(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))))
        side = min(max(side, lo), hi)
        bc = tuple(_uniform(seed, 5 * p + 1 + k) for k in range(4))
        out.append(Problem(side, side, max_sweeps, check_every=check_every, tol=tol, bc=bc))
    return out


@dataclass
class Candidate:
    chare_side: int
    pes_per_sm: int
    ring_bytes: int
    ms: float = float("inf")
    glups: float = 0.0

    def runtime_config(self) -> dict:
        cfg = dict(pes_per_sm=self.pes_per_sm, threads_per_pe=512 // self.pes_per_sm,
                   ring_bytes=self.ring_bytes)
        if self.ring_bytes < (4 << 20):
            cfg["max_msg_bytes"] = min(self.ring_bytes // 4, (1 << 20) + 64)
        return cfg

    def key(self) -> str:
        return f"side{self.chare_side}_pes{self.pes_per_sm}_ring{self.ring_bytes >> 10}k"


@dataclass
class TuneResult:
    best: Candidate
    tried: list = field(default_factory=list)
    seconds: float = 0.0

    def as_dict(self) -> dict:
        return {"chosen": self.best.key(), "chare_side": self.best.chare_side,
                "pes_per_sm": self.best.pes_per_sm, "ring_bytes": self.best.ring_bytes,
                "tried": {c.key(): round(c.glups, 1) for c in self.tried},
                "tune_s": round(self.seconds, 2)}


def default_candidates() -> list[Candidate]:
    return [Candidate(s, p, r) for s, p, r in
            itertools.product((64, 128, 256), (1, 2, 4), (1 << 20, 4 << 20))]


def time_set(problems, dtype: str, chare_side: int, runs: int = 2, warmup: int = 1,
             use_graph: bool = True) -> float:
    """Mean ms of `runs` graph-replayed launches of the whole set."""
    with Jacobi2D(problems, dtype=dtype, chare_side=chare_side, use_graph=use_graph) as j:
        for _ in range(warmup):
            j.run()
        ts = [j.run() for _ in range(runs)]
    return float(np.mean(ts))


def autotune(problems, dtype: str = "f64", candidates=None, runs: int = 2,
             device: int = 0) -> TuneResult:
    """Times the set under every candidate and returns the fastest. Leaves
    the runtime initialised with the winner's configuration."""
    t0 = time.perf_counter()
    cands = list(candidates or default_candidates())
    lups = sum(p.nx * p.ny * p.max_sweeps for p in problems)
    for c in cands:
        try:
            Runtime(device=device, **c.runtime_config())
            c.ms = time_set(problems, dtype, c.chare_side, runs=runs)
            c.glups = lups / (c.ms * 1e-3) / 1e9
        except CharmingError:
            c.ms, c.glups = float("inf"), 0.0  # a configuration the device cannot run
    best = min(cands, key=lambda c: c.ms)
    Runtime(device=device, **best.runtime_config())
    return TuneResult(best, cands, time.perf_counter() - t0)


def save_choice(path: str, key: str, result: TuneResult) -> None:
    """Records a tuning result under `key` (problem set, dtype, device) in a
    JSON file, so a later process can reuse it."""
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data[key] = result.as_dict()
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
