"""CPU model of the messaging semantics. TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker; the product never calls it.

It restates, in plain numpy / Python:

* the seeded generators shared with the GPU programs (SplitMix64 finaliser,
  payload word stream, position-dependent checksum);
* the fan-out workload (destinations, per-receiver expected counts per refnum,
  payload checksums) and a checker for the GPU's delivery log;
* an event model of refnum matching, stash and revive, following the
  reference: ``include/chare.h:181-195`` (deliver iff the message refnum is -1
  or equals the chare's), ``src/comm/get/get.cu:422-444`` (park mismatches),
  ``src/comm/get/get.cu:1316-1345`` (``set_refnum`` revives parked messages
  with the new refnum).  Per-(sender, receiver) FIFO order is stronger than
  the reference guarantees (its slot scan reorders, ``get.cu:234-259`` and
  ``:337-344``); the model and the runtime both deliver in send order.

Parity status: the reference has no golden vectors or tests for messaging;
its observable behaviour is the example output (hello chain,
``examples/hello/hello.cu:38-51``; refnum order "1" then "0",
``examples/refnum/refnum.cu:27-53``), which the model reproduces as known
answers.  The generators are pinned against the published SplitMix64
sequence.
"""
from __future__ import annotations

from collections import defaultdict, deque
from dataclasses import dataclass, field

import numpy as np

M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15
STREAM_K = 0xD1B54A32D192ED03
CHECK_K = 0xA0761D6478BD642F


# ---------------------------------------------------------------------------
# generators (restated from charming_b200/csrc/apps/suite.cuh)
# ---------------------------------------------------------------------------
def mix64(z):
    """SplitMix64 finaliser of (z + golden); numpy uint64 arrays or ints."""
    if isinstance(z, (int, np.integer)):
        z = (int(z) + GOLDEN) & M64
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def splitmix64_sequence(seed: int, n: int) -> list[int]:
    """The standard SplitMix64 generator: output k = mix64(seed + k*golden)."""
    return [mix64((seed + k * GOLDEN) & M64) for k in range(n)]


def gen_words(seed: int, stream: int, n: int) -> np.ndarray:
    """Payload word stream: mix64(seed ^ stream*K ^ j*golden), j = 0..n-1."""
    j = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed & M64) ^ np.uint64((stream * STREAM_K) & M64) ^ (j * np.uint64(GOLDEN))
    return mix64(x)


def checksum(data: bytes | np.ndarray) -> int:
    """sum_i mix64(w_i ^ (i+1)*K) mod 2^64, xor len; w_i little-endian words."""
    b = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data.view(np.uint8)
    n = b.size
    nw = (n + 7) // 8
    padded = np.zeros(nw * 8, dtype=np.uint8)
    padded[:n] = b
    w = padded.view("<u8").astype(np.uint64)
    i = np.arange(nw, dtype=np.uint64)
    with np.errstate(over="ignore"):
        terms = mix64(w ^ ((i + np.uint64(1)) * np.uint64(CHECK_K)))
        s = int(np.sum(terms, dtype=np.uint64)) if nw else 0
    return (s & M64) ^ n


def payload_bytes(seed: int, stream: int, nbytes: int) -> bytes:
    nw = (nbytes + 7) // 8
    return gen_words(seed, stream, nw).astype("<u8").tobytes()[:nbytes]


# ---------------------------------------------------------------------------
# pingpong
# ---------------------------------------------------------------------------
def pingpong_checksums(seed: int, sizes) -> np.ndarray:
    """[chare][size] checksum of chare's payload prefix (chare 0 and 1)."""
    out = np.zeros((2, len(sizes)), dtype=np.uint64)
    for who in (0, 1):
        full = payload_bytes(seed, who, int(max(sizes)))
        for s, n in enumerate(sizes):
            out[who, s] = checksum(full[: int(n)])
    return out


# ---------------------------------------------------------------------------
# fan-out
# ---------------------------------------------------------------------------
def fanout_destinations(n: int, msgs: int, seed: int) -> np.ndarray:
    """dst[s, k] = mix64(seed ^ ((s*msgs + k + 1) * golden)) % n."""
    ids = np.arange(n * msgs, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed & M64) ^ ((ids + np.uint64(1)) * np.uint64(GOLDEN))
    return (mix64(x) % np.uint64(n)).astype(np.int64).reshape(n, msgs)


def fanout_expected_counts(n: int, msgs: int, seed: int) -> np.ndarray:
    """counts[d, k] = number of messages with refnum k addressed to chare d."""
    dst = fanout_destinations(n, msgs, seed)
    counts = np.zeros((n, msgs), dtype=np.int64)
    for k in range(msgs):
        np.add.at(counts[:, k], dst[:, k], 1)
    return counts


def fanout_payload(seed: int, n: int, msgs: int, payload: int, s: int, k: int, mode: int) -> bytes:
    stream = s * msgs + k
    w = gen_words(seed, stream, (payload + 7) // 8)
    w[0] = np.uint64(s | (k << 32))
    w[1] = np.uint64((k if mode else -1) & 0xFFFFFFFF)
    return w.astype("<u8").tobytes()[:payload]


def fanout_checksums(n: int, msgs: int, payload: int, seed: int, mode: int) -> np.ndarray:
    """Vectorised checksum of every fan-out payload, [n, msgs] uint64."""
    nw = payload // 8
    sid = np.arange(n * msgs, dtype=np.uint64)
    j = np.arange(nw, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = (np.uint64(seed & M64) ^ (sid[:, None] * np.uint64(STREAM_K))) ^ (j[None, :] * np.uint64(GOLDEN))
        w = mix64(x)
        s = sid // np.uint64(msgs)
        k = sid % np.uint64(msgs)
        w[:, 0] = s | (k << np.uint64(32))
        w[:, 1] = k if mode else np.uint64(0xFFFFFFFF)
        terms = mix64(w ^ ((j[None, :] + np.uint64(1)) * np.uint64(CHECK_K)))
        tot = np.sum(terms, axis=1, dtype=np.uint64)
    return (tot ^ np.uint64(payload)).reshape(n, msgs)


@dataclass
class LogCheck:
    ok: bool
    errors: list = field(default_factory=list)
    delivered: int = 0


def check_fanout_log(log: np.ndarray, n: int, msgs: int, payload: int, seed: int, mode: int,
                     max_errors: int = 20) -> LogCheck:
    """Checks a delivery log (records of 8 x uint32: dst, src, k, refnum field,
    seq at dst, checksum lo, checksum hi, receiver refnum at delivery)
    against the model: exact delivery set, checksums, per-pair FIFO, and (mode
    1) refnum matching with monotone receiver refnums."""
    errs = []
    log = np.asarray(log, dtype=np.uint32).reshape(-1, 8)
    total = n * msgs
    if log.shape[0] != total:
        errs.append(f"delivered {log.shape[0]} messages, expected {total}")
    dst_exp = fanout_destinations(n, msgs, seed)
    cs_exp = fanout_checksums(n, msgs, payload, seed, mode)
    dst, src, k = log[:, 0].astype(np.int64), log[:, 1].astype(np.int64), log[:, 2].astype(np.int64)
    ref_field = log[:, 3].astype(np.int64)
    seq = log[:, 4].astype(np.int64)
    cs = log[:, 5].astype(np.uint64) | (log[:, 6].astype(np.uint64) << np.uint64(32))
    rcv_ref = log[:, 7].astype(np.int64)
    if np.any((src < 0) | (src >= n) | (k < 0) | (k >= msgs)):
        errs.append("record with out-of-range src or k")
        return LogCheck(False, errs, int(log.shape[0]))
    ids = src * msgs + k
    seen = np.bincount(ids, minlength=total)
    if np.any(seen != 1):
        bad = np.nonzero(seen != 1)[0][:5]
        errs.append(f"messages delivered != once: ids {bad.tolist()} counts {seen[bad].tolist()}")
    wrong_dst = np.nonzero(dst_exp[src, k] != dst)[0]
    if wrong_dst.size:
        errs.append(f"{wrong_dst.size} messages delivered to the wrong chare")
    wrong_cs = np.nonzero(cs_exp[src, k] != cs)[0]
    if wrong_cs.size:
        errs.append(f"{wrong_cs.size} payload checksum mismatches")
    exp_ref = k if mode else np.full_like(k, 0xFFFFFFFF)
    if np.any(ref_field != exp_ref):
        errs.append("refnum field in payload differs from the sent refnum")
    # per-receiver sequence numbers are a permutation of 0..count-1
    order = np.lexsort((seq, dst))
    d_sorted, s_sorted = dst[order], seq[order]
    starts = np.r_[0, np.nonzero(np.diff(d_sorted))[0] + 1]
    for a, b in zip(starts, np.r_[starts[1:], d_sorted.size]):
        if not np.array_equal(s_sorted[a:b], np.arange(b - a)):
            errs.append(f"receiver {int(d_sorted[a])}: sequence numbers not 0..{b - a - 1}")
            if len(errs) > max_errors:
                break
    # per-(src, dst) FIFO: in delivery order at dst, k increases
    order = np.lexsort((seq, src, dst))
    ds, ss, ks = dst[order], src[order], k[order]
    same_pair = (ds[1:] == ds[:-1]) & (ss[1:] == ss[:-1])
    fifo_bad = np.nonzero(same_pair & (ks[1:] <= ks[:-1]))[0]
    if fifo_bad.size:
        errs.append(f"{fifo_bad.size} per-pair FIFO violations")
    if mode:
        if np.any(rcv_ref != k):
            errs.append(f"{int(np.sum(rcv_ref != k))} deliveries with refnum != receiver refnum")
        order = np.lexsort((seq, dst))
        dd, kk = dst[order], k[order]
        mono_bad = np.nonzero((dd[1:] == dd[:-1]) & (kk[1:] < kk[:-1]))[0]
        if mono_bad.size:
            errs.append(f"{mono_bad.size} deliveries out of refnum order at a receiver")
    return LogCheck(not errs, errs[:max_errors], int(log.shape[0]))


# ---------------------------------------------------------------------------
# event model of refnum matching / stash / revive (one receiving PE)
# ---------------------------------------------------------------------------
@dataclass
class Msg:
    chare: int
    refnum: int
    payload: object = None


class ReceiverModel:
    """Delivery order at one PE given its inbox arrival order.

    ``on_deliver(model, msg)`` is the entry method; it may call
    ``model.set_refnum(chare, v)``.  Semantics: a message is delivered when
    its refnum is -1 or equals the chare's refnum, else parked; after an
    entry method, parked messages whose refnum now matches are delivered in
    arrival order before the next inbox message (re-checked at delivery).
    """

    def __init__(self, refnums: dict[int, int], on_deliver):
        self.refnum = dict(refnums)
        self.on_deliver = on_deliver
        self.stash: list[Msg] = []
        self.ready: deque[Msg] = deque()
        self.delivered: list[Msg] = []
        self._dirty = False

    def set_refnum(self, chare: int, v: int) -> None:
        self.refnum[chare] = v
        self._dirty = True

    def _matches(self, m: Msg) -> bool:
        return m.refnum == -1 or m.refnum == self.refnum.get(m.chare, -1)

    def _revive(self) -> None:
        if not self._dirty:
            return
        self._dirty = False
        keep = []
        for m in self.stash:
            (self.ready.append if self._matches(m) else keep.append)(m)
        self.stash = keep

    def _run(self, m: Msg) -> None:
        self.delivered.append(m)
        self.on_deliver(self, m)
        self._revive()

    def arrive(self, m: Msg) -> None:
        while self.ready:
            r = self.ready.popleft()
            if self._matches(r):
                self._run(r)
            else:
                self.stash.append(r)
        if self._matches(m):
            self._run(m)
        else:
            self.stash.append(m)
        while self.ready:
            r = self.ready.popleft()
            if self._matches(r):
                self._run(r)
            else:
                self.stash.append(r)


def refnum_scenario(reversed_order: bool = False) -> list[int]:
    """examples/refnum/refnum.cu:27-53: chare 1 starts at refnum 1; chare 0
    sends refnum 1 then 0 (or 0 then 1 when reversed); on each delivery chare
    1 records the payload and sets its refnum to 0. Returns delivered refnums."""
    sends = [0, 1] if reversed_order else [1, 0]

    def em(model, m):
        model.set_refnum(1, 0)

    rm = ReceiverModel({1: 1}, em)
    for r in sends:
        rm.arrive(Msg(1, r, r))
    return [m.payload for m in rm.delivered]


def hello_chain(n_pes: int) -> list[int]:
    """examples/hello/hello.cu:32-52: chare i receives i (2*n_pes chares)."""
    n = 2 * n_pes
    received = []
    v = 0
    for i in range(n):
        received.append(v)
        v += 1
    return received
