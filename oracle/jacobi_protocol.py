"""CPU model of the Jacobi2d chare protocol. TEST INFRASTRUCTURE ONLY.

Restates the state machine of charming_b200/csrc/apps/jacobi_chare.cuh
(halos per sweep with parity ghost buffers, the binary residual tree, the
stop decision applied one check period later, and with two_phase the
exchange of ghost depth > 1: left/right halos first, top/bottom halos sent
once the left/right ones of the same pass are in, so that they carry the
corners) with messages delivered in
per-pair FIFO order but otherwise in a random interleaving, and checks its
invariants: a halo never arrives more than one sweep ahead, a sweep never
starts without all halos of its sweep, every chare stops at the same sweep,
no tree message finds its slot occupied, and once every chare has finished
no message is left in flight and none reached a finished chare (a chare at
max_sweeps waits for the decision of the last check first).
"""
from __future__ import annotations

import random
from collections import deque
from dataclasses import dataclass, field


@dataclass
class Chare:
    idx: int
    nbrs: list
    xn: list     # left/right neighbours (the first phase of a two-phase exchange)
    parent: int
    children: list
    rank: int
    iter: int = 0
    sent: int = -1
    started: bool = False
    got: list = field(default_factory=lambda: [0, 0])
    gotx: list = field(default_factory=lambda: [0, 0])
    sent_y: int = -1
    halo_seen: dict = field(default_factory=dict)
    done: bool = False
    waiting: bool = False
    have_own: bool = False
    own: float = 0.0
    child_got: list = field(default_factory=lambda: [False, False])
    child_val: list = field(default_factory=lambda: [0.0, 0.0])
    decided: int = -1
    stop_check: int = -1
    res0: float = 0.0


class ProtocolError(AssertionError):
    pass


class Sim:
    def __init__(self, px, py, K, max_sweeps, stop_at_check, seed=0, two_phase=False):
        self.rng = random.Random(seed)
        self.two_phase = two_phase
        self.K, self.max = K, max_sweeps
        self.stop_at_check = stop_at_check  # residual decision that says stop
        n = px * py
        self.ch = []
        for r in range(n):
            cy, cx = divmod(r, px)
            nb = []
            if cy > 0: nb.append(r - px)
            if cy < py - 1: nb.append(r + px)
            xn = []
            if cx > 0: xn.append(r - 1)
            if cx < px - 1: xn.append(r + 1)
            kids = [k for k in (2 * r + 1, 2 * r + 2) if k < n]
            self.ch.append(Chare(r, nb + xn, xn, (r - 1) // 2 if r > 0 else -1, kids, r))
        self.queues = {}  # (src, dst) -> deque of messages (per-pair FIFO)
        self.finished_at = {}

    def send(self, src, dst, msg):
        self.queues.setdefault((src, dst), deque()).append(msg)

    # ---- the chare logic (mirrors jacobi_chare.cuh) ----
    def pump(self, c):
        while True:
            if c.done or c.waiting:
                return
            if c.sent < c.iter:
                K = self.K
                if c.iter >= self.max:
                    if K > 0 and self.max > 0 and c.decided < (self.max - 1) // K:
                        c.waiting = True
                        return
                    return self.finish(c)
                if K > 0 and c.iter >= K and c.iter % K == 0 and c.decided < c.iter // K - 1:
                    c.waiting = True
                    return
                if K > 0 and c.iter >= K and c.iter % K == 0 and 0 <= c.stop_check <= c.iter // K - 1:
                    return self.finish(c)
                c.sent = c.iter
                for nb in (c.xn if self.two_phase else c.nbrs):
                    self.send(c.idx, nb, ("halo", c.iter, "x" if self.two_phase else "all"))
                continue
            if self.two_phase and c.sent_y < c.iter and c.gotx[c.iter & 1] == len(c.xn):
                c.sent_y = c.iter
                for nb in c.nbrs:
                    if nb not in c.xn:
                        self.send(c.idx, nb, ("halo", c.iter, "y"))
                continue
            if c.nbrs and c.got[c.iter & 1] == len(c.nbrs) and (not self.two_phase or c.sent_y == c.iter):
                self.advance(c)
                continue
            return

    def advance(self, c):
        if c.got[c.iter & 1] != len(c.nbrs):
            raise ProtocolError(f"chare {c.idx} sweeps {c.iter} without all halos")
        K = self.K
        resid = K > 0 and c.iter % K == 0
        chk = c.iter // K if K else 0
        if self.two_phase and c.sent_y != c.iter:
            raise ProtocolError(f"chare {c.idx} sweeps {c.iter} before its top/bottom halos went out")
        c.got[c.iter & 1] = 0
        c.gotx[c.iter & 1] = 0
        c.iter += 1
        if resid:
            if c.have_own:
                raise ProtocolError(f"chare {c.idx}: own partial of an earlier check not sent")
            c.own, c.have_own = 1.0, True
            self.tree_try_forward(c, chk)

    def tree_try_forward(self, c, chk):
        complete = c.have_own and all(c.child_got[k] for k in range(len(c.children)))
        if not complete:
            return
        total = c.own + sum(c.child_val[k] for k in range(len(c.children)))
        c.have_own = False
        c.child_got = [False, False]
        if c.parent >= 0:
            self.send(c.idx, c.parent, ("partial", chk, (c.rank - 1) % 2, total))
        else:
            self.apply_decision(c, chk, chk >= self.stop_at_check)

    def apply_decision(self, c, chk, stop):
        c.decided = max(c.decided, chk)
        if stop and c.stop_check < 0:
            c.stop_check = chk
        resume = c.waiting
        c.waiting = False
        for k in c.children:
            self.send(c.idx, k, ("decision", chk, stop))
        if resume:
            self.pump(c)

    def finish(self, c):
        c.done = True
        self.finished_at[c.idx] = c.iter

    def deliver(self, c, msg):
        if msg[0] == "start":
            c.started = True
            return self.pump(c)
        if c.done:
            raise ProtocolError(f"chare {c.idx} got {msg[0]} after it finished")
        if msg[0] == "halo":
            k = msg[1]
            if k not in (c.iter, c.iter + 1):
                raise ProtocolError(f"chare {c.idx} at {c.iter} got halo of sweep {k}")
            c.got[k & 1] += 1
            if msg[2] == "x":
                c.gotx[k & 1] += 1
            if c.got[k & 1] > len(c.nbrs) or c.gotx[k & 1] > len(c.xn):
                raise ProtocolError(f"chare {c.idx}: too many halos of parity {k & 1}")
            if c.started:
                self.pump(c)
        elif msg[0] == "partial":
            _, chk, slot, val = msg
            if slot >= len(c.children) or c.child_got[slot]:
                raise ProtocolError(f"chare {c.idx}: partial slot {slot} of check {chk} busy")
            c.child_val[slot], c.child_got[slot] = val, True
            self.tree_try_forward(c, chk)
        elif msg[0] == "decision":
            self.apply_decision(c, msg[1], msg[2])

    def run(self, max_steps=10_000_000):
        for c in self.ch:
            self.send(-1, c.idx, ("start",))
        steps = 0
        while len(self.finished_at) < len(self.ch):
            live = [k for k, q in self.queues.items() if q]
            if not live:
                raise ProtocolError("deadlock: no message in flight, chares not done")
            src, dst = self.rng.choice(live)
            msg = self.queues[(src, dst)].popleft()
            self.deliver(self.ch[dst], msg)
            steps += 1
            if steps > max_steps:
                raise ProtocolError("no progress")
        left = sum(len(q) for q in self.queues.values())
        if left:
            raise ProtocolError(f"{left} messages in flight after every chare finished")
        ends = set(self.finished_at.values())
        if len(ends) != 1:
            raise ProtocolError(f"chares stopped at different sweeps: {sorted(ends)}")
        return ends.pop()
