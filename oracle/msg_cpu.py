"""CPU baseline of the messaging benchmarks (test infrastructure, timed
beside the GPU numbers; never part of the product): ctypes binding of liboracle_msg.so (msg_cpu.c), the GPU's
fan-out and pingpong workloads on host threads with one MPSC inbox each."""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(os.path.join(_HERE, "liboracle_msg.so"))
        _lib.cpu_fanout.restype = C.c_double
        _lib.cpu_fanout.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int,
                                    C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        _lib.cpu_pingpong.restype = C.c_double
        _lib.cpu_pingpong.argtypes = [C.c_uint64, C.c_int, C.c_uint64]
    return _lib


def fanout(n: int, msgs: int, payload: int, seed: int, threads: int) -> tuple[float, int]:
    """Seconds of the exchange and messages delivered."""
    d, cs = C.c_uint64(0), C.c_uint64(0)
    s = lib().cpu_fanout(n, msgs, payload, seed, threads, C.byref(d), C.byref(cs))
    if s < 0:
        raise ValueError("cpu_fanout: bad arguments")
    return s, d.value


def pingpong_oneway_s(nbytes: int, round_trips: int, seed: int = 1) -> float:
    return lib().cpu_pingpong(nbytes, round_trips, seed)
