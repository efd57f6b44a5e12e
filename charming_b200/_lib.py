"""ctypes binding of libcharming_b200.so (include/charming_c.h).

The shared library is built in-tree (charming_b200/lib/) by
``charming_b200.build.build_all()``.  Loading fails loudly when it is
missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
# CHARMING_CHECKED=1 selects the build with invariant checks (make CHECKS=1).
LIB_PATH = os.path.join(LIB_DIR, "libcharming_b200_checked.so"
                        if os.environ.get("CHARMING_CHECKED") == "1" else "libcharming_b200.so")
# The multi-GPU build (runs over several GPUs, or virtual GPUs on one):
# loaded instead when the first runtime of the process asks for several
# GPUs, or with CHARMING_MULTI_GPU=1.
MULTI_LIB_PATH = os.path.join(LIB_DIR, "libcharming_b200_multi.so")
# CHARMING_LIB: path of another build of the same library (e.g. one compiled
# with a different register limit); it is used whatever the runtime asks for.
LIB_OVERRIDE = os.environ.get("CHARMING_LIB")
LIB_PATH = LIB_OVERRIDE or LIB_PATH

u64 = C.c_uint64
i32 = C.c_int
f64 = C.c_double
vp = C.c_void_p

# status codes (charming_c.h)
STATUS = {
    0: "OK", 1: "RING_FULL", 2: "STASH_FULL", 3: "BAD_TARGET", 4: "BARRIER_TIMEOUT",
    5: "IDLE_TIMEOUT", 6: "DEADLINE", 7: "BAD_MSG", 8: "MSG_TOO_LARGE", 9: "HOST_STOP",
    10: "TOO_MANY_TYPES", 11: "TOO_MANY_EMS", 12: "PIPELINE", 13: "LAUNCH", 14: "CONFIG",
    15: "CUDA", 16: "NOT_INIT", 17: "NO_MEMORY", 18: "APP", 19: "TOO_MANY_WAITS",
}
F64, F32 = 0, 1


class Config(C.Structure):
    _fields_ = [
        ("device", i32), ("pes_per_sm", i32), ("threads_per_pe", i32), ("n_pes", i32),
        ("ring_bytes", u64), ("max_msg_bytes", u64), ("stash_bytes", u64),
        ("stash_entries", i32), ("heap_bytes", u64), ("stack_bytes", u64),
        ("deadline_s", f64), ("idle_timeout_s", f64), ("free_chares_at_exit", i32),
        ("verbose", i32), ("gpu_level", i32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("n_pes", i32), ("n_sms", i32), ("threads_per_pe", i32), ("smem_bytes_per_pe", i32),
        ("smem_scratch_bytes", i32), ("regs_per_thread", i32), ("ring_bytes", u64),
        ("max_msg_bytes", u64), ("device_bytes", u64), ("stack_bytes", u64),
        ("local_bytes", u64), ("n_blocks", i32), ("gpu_level", i32), ("n_devs", i32), ("my_dev", i32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("delivered", u64), ("sent", u64), ("stashed", u64), ("revived", u64),
        ("bytes_sent", u64), ("idle_polls", u64), ("space_waits", u64),
        ("kernel_ms", f64), ("loop_ms", f64), ("main_ms", f64), ("status", i32), ("err_pe", i32),
        ("err_info0", i32), ("err_info1", i32), ("idle_ms", f64), ("em_ms", f64),
        ("deferred", u64), ("ticket_ms", f64), ("space_ms", f64), ("batched", u64),
    ]


class JacobiProblem(C.Structure):
    _fields_ = [
        ("nx", i32), ("ny", i32), ("px", i32), ("py", i32), ("max_sweeps", i32),
        ("check_every", i32), ("tol", f64), ("bc", f64 * 4),
    ]


class JacobiOptions(C.Structure):
    _fields_ = [
        ("dtype", i32), ("chare_side", i32), ("tile_w", i32), ("pipeline", i32),
        ("use_graph", i32), ("balance", i32), ("halo_mode", i32), ("depth", i32),
    ]


class JacobiResult(C.Structure):
    _fields_ = [("sweeps", i32), ("checks", i32), ("res0", f64), ("res_last", f64)]


class JacobiInfo(C.Structure):
    _fields_ = [
        ("n_problems", i32), ("n_chares", i32), ("max_chares_per_pe", i32),
        ("interior_points", u64), ("grid_bytes", u64), ("halo_msgs_per_sweep", u64),
        ("last_run_ms", f64), ("sweep_ms_max", f64), ("sweep_ms_mean", f64),
        ("send_ms_mean", f64), ("halo_ms_mean", f64), ("send_reserve_ms_mean", f64),
        ("send_publish_ms_mean", f64), ("send_setup_ms_mean", f64),
    ]


class PingpongResult(C.Structure):
    _fields_ = [("size", u64), ("oneway_us", f64), ("oneway_cycles", f64),
                ("checksum_errors", u64)]


class ServeConfig(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", u64), ("max_inflight", i32), ("workers_per_pe", i32),
        ("chare_side", i32), ("dtype", i32), ("deadline_s", f64),
    ]


class ServeCompletion(C.Structure):
    _fields_ = [
        ("tag", u64), ("status", i32), ("sweeps", i32), ("res0", f64), ("res_last", f64),
        ("submit_s", f64), ("admit_s", f64), ("done_s", f64),
    ]


class ServeStats(C.Structure):
    _fields_ = [
        ("submitted", u64), ("admitted", u64), ("completed", u64), ("peak_bytes", u64),
        ("peak_inflight", i32), ("busy_s", f64),
    ]


# Several GPUs (charming_devices): the host's allgather and barrier.
ALLGATHER_FN = C.CFUNCTYPE(i32, vp, vp, vp, C.c_size_t)
BARRIER_FN = C.CFUNCTYPE(i32, vp)


class Devices(C.Structure):
    _fields_ = [
        ("rank", i32), ("world", i32), ("virtual_devs", i32), ("reserved", i32),
        ("allgather", ALLGATHER_FN), ("barrier", BARRIER_FN), ("ctx", vp),
    ]


# (name, restype, argtypes) for every entry point of charming_c.h
SIGNATURES = [
    ("charming_default_config", None, [C.POINTER(Config)]),
    ("charming_init", i32, [C.POINTER(Config)]),
    ("charming_init_devices", i32, [C.POINTER(Config), C.POINTER(Devices)]),
    ("charming_run", i32, [i32, C.POINTER(C.c_char_p)]),
    ("charming_fini", i32, []),
    ("charming_timer_start", i32, []),
    ("charming_timer_stop", i32, [C.POINTER(f64)]),
    ("charming_get_info", i32, [C.POINTER(Info)]),
    ("charming_last_stats", i32, [C.POINTER(Stats)]),
    ("charming_status_string", C.c_char_p, [i32]),
    ("charming_last_error", C.c_char_p, []),
    ("charming_jacobi2d_create", i32, [C.POINTER(JacobiProblem), i32, C.POINTER(JacobiOptions), C.POINTER(vp)]),
    ("charming_jacobi2d_init", i32, [vp]),
    ("charming_jacobi2d_load", i32, [vp, i32, vp]),
    ("charming_jacobi2d_run", i32, [vp]),
    ("charming_jacobi2d_run_n", i32, [vp, i32, C.POINTER(f64)]),
    ("charming_jacobi2d_store", i32, [vp, i32, vp]),
    ("charming_jacobi2d_result", i32, [vp, i32, C.POINTER(JacobiResult)]),
    ("charming_jacobi2d_get_info", i32, [vp, C.POINTER(JacobiInfo)]),
    ("charming_jacobi2d_destroy", i32, [vp]),
    ("charming_jacobi2d_sweeps_noalloc", i32, [i32, i32, i32, i32, vp, vp]),
    ("charming_jacobi1d", i32, [i32, i32, i32, C.POINTER(f64), C.POINTER(f64)]),
    ("charming_pingpong", i32, [C.POINTER(u64), i32, i32, i32, u64, i32, C.POINTER(PingpongResult), C.POINTER(i32)]),
    ("charming_fanout", i32, [i32, i32, i32, u64, i32, C.POINTER(C.c_uint32), u64, C.POINTER(u64), C.POINTER(f64)]),
    ("charming_hello", i32, [C.POINTER(i32), i32, C.POINTER(i32)]),
    ("charming_refnum", i32, [C.POINTER(i32), i32, C.POINTER(i32)]),
    ("charming_refnum_reversed", i32, [C.POINTER(i32), i32, C.POINTER(i32)]),
    ("charming_async_wait_chain", i32, [i32, i32, C.POINTER(i32), i32]),
    ("charming_sm_pingpong", i32, [i32, i32, C.POINTER(f64), C.POINTER(f64), C.POINTER(i32)]),
    ("charming_sweep_bench", i32, [i32, i32, i32, i32, i32, i32, i32, C.POINTER(f64)]),
    ("charming_jacobi2d_decomp1d", i32, [i32, i32, i32, i32, i32, C.POINTER(C.c_float), C.POINTER(f64)]),
    ("charming_jacobi3d", i32, [i32, i32, i32, i32, C.POINTER(f64), C.POINTER(f64)]),
    ("charming_jacobi2d_solve_stream", i32, [vp, i32, i32, C.POINTER(vp), C.POINTER(vp), C.POINTER(f64)]),
    ("charming_user_heap_check", i32, [i32, i32, i32, u64, C.POINTER(u64)]),
    ("charming_serve_start", i32, [C.POINTER(ServeConfig), C.POINTER(vp)]),
    ("charming_serve_submit", i32, [vp, C.POINTER(JacobiProblem), u64]),
    ("charming_serve_poll", i32, [vp, C.POINTER(ServeCompletion), i32, C.POINTER(i32)]),
    ("charming_serve_fetch", i32, [vp, u64, vp]),
    ("charming_serve_release", i32, [vp, u64]),
    ("charming_serve_stop", i32, [vp, C.POINTER(ServeStats)]),
]

_lib = None
_lock = threading.Lock()


def load(multi: bool = False) -> C.CDLL:
    """Loads libcharming_b200.so (multi: the multi-GPU build); raises if it
    has not been built. One build per process: asking for several GPUs
    after the single-GPU build was loaded raises."""
    global _lib
    multi = multi or os.environ.get("CHARMING_MULTI_GPU") == "1"
    with _lock:
        if _lib is not None:
            if multi and not _lib.multi_gpu:
                raise RuntimeError("this process loaded the single-GPU build of the library; several "
                                   "GPUs need the multi-GPU build (set CHARMING_MULTI_GPU=1, or create "
                                   "the multi-GPU runtime first)")
            return _lib
        path = MULTI_LIB_PATH if (multi and not LIB_OVERRIDE) else LIB_PATH
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build it with charming_b200.build.build_all() "
                "(there is no CPU fallback)")
        lib = C.CDLL(path, mode=C.RTLD_GLOBAL)
        lib.multi_gpu = multi or path == MULTI_LIB_PATH
        missing = []
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name, None)
            if fn is None:
                missing.append(name)
                continue
            fn.restype = res
            fn.argtypes = args
        lib.missing_symbols = missing
        _lib = lib
        return lib


class CharmingError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        lib = _lib
        text = lib.charming_status_string(code).decode() if lib else STATUS.get(code, "?")
        detail = lib.charming_last_error().decode() if lib else ""
        super().__init__(f"{what}: status {code} ({STATUS.get(code, '?')}: {text}) {detail}".strip())


def check(code: int, what: str = "") -> int:
    if code != 0:
        raise CharmingError(code, what)
    return code
