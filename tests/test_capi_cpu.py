"""CPU tests of the C ABI library: it loads and exports every declared symbol."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        if 'extern "C"' not in text:
            continue
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(charming_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from charming_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert not lib.missing_symbols


def test_multi_gpu_build_exports_every_declared_symbol():
    # the multi-GPU build (several GPUs, one process each, or virtual GPUs)
    # is the same C ABI; a fresh process, since one process holds one build
    # (a second copy's CUDA registrations clash with the first's)
    import json
    import subprocess
    import sys
    code = ("import ctypes, json, sys; sys.path.insert(0, %r); from tests.test_capi_cpu import declared_functions; "
            "lib = ctypes.CDLL(%r); print(json.dumps([n for n in declared_functions() if not hasattr(lib, n)]))"
            % (ROOT, os.path.join(ROOT, "charming_b200", "lib", "libcharming_b200_multi.so")))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert json.loads(r.stdout.strip().splitlines()[-1]) == []


def test_bindings_cover_every_declared_symbol():
    from charming_b200 import _lib
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_status_strings_and_default_config():
    from charming_b200 import _lib
    lib = _lib.load()
    assert lib.charming_status_string(0) == b"ok"
    assert b"stash" in lib.charming_status_string(2)
    cfg = _lib.Config()
    lib.charming_default_config(C.byref(cfg))
    assert cfg.threads_per_pe == 512 and cfg.ring_bytes == 4 << 20
    assert cfg.pes_per_sm == 1 and cfg.stash_entries == 4096


def test_struct_sizes_match_header():
    # Layout of the C structs as compiled (sizeof probes built into the .so
    # would need a GPU-free entry point; compare against the ctypes layout of
    # the fields declared in the header instead).
    from charming_b200 import _lib
    assert C.sizeof(_lib.JacobiProblem) == 4 * 6 + 8 * 5
    assert C.sizeof(_lib.Config) == 96  # gpu_level + tail padding


def test_reference_examples_built():
    d = os.path.join(ROOT, "build", "ref_examples")
    from charming_b200 import build
    if not os.path.isdir(os.path.join(build.REFERENCE, "examples")):
        pytest.skip("reference tree not present")
    for ex in ("hello", "refnum", "pingpong"):
        assert os.path.exists(os.path.join(d, ex)), ex
        assert os.path.exists(os.path.join(d, f"{ex}_multi")), ex  # against libcharming_multi.a
    # pingpong's GPU-level branch (the reference's default build) compiles and
    # links unchanged too; it places its two chares with block_map[0] and
    # block_map[n_pes / 2], so it needs two PEs, i.e. two GPUs, in that mode
    assert os.path.exists(os.path.join(d, "pingpong_gpu_level"))
