"""The device API forms of the reference's headers compile against include/
and link against libcharming.a (nvcc cross-compiles for sm_100a without a
GPU): the const message invoke overloads, malloc_user / free_user and
async_wait (tests/compile/api_forms.cu), and a GPU-level program
(tests/compile/gpu_level_forms.cu, -DCHARMING_GPU_LEVEL)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARCH = "-gencode arch=compute_100a,code=sm_100a"


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not installed")
def test_reference_api_forms_compile_and_link(tmp_path):
    lib = os.path.join(ROOT, "charming_b200", "lib", "libcharming.a")
    assert os.path.exists(lib), "build the runtime first (__graft_entry__.build)"
    src = os.path.join(ROOT, "tests", "compile", "api_forms.cu")
    obj, exe = tmp_path / "api_forms.o", tmp_path / "api_forms"
    inc = os.path.join(ROOT, "include")
    r = subprocess.run(f"nvcc -std=c++17 {ARCH} -rdc=true -I{inc} -c {src} -o {obj}", shell=True,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run(f"nvcc {ARCH} -rdc=true -Xnvlink -suppress-stack-size-warning -o {exe} {obj} "
                       f"{lib} -lcudart", shell=True, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    assert exe.exists()


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not installed")
def test_gpu_level_program_compiles_links_and_asks_for_the_mode(tmp_path):
    lib = os.path.join(ROOT, "charming_b200", "lib", "libcharming.a")
    assert os.path.exists(lib), "build the runtime first (__graft_entry__.build)"
    src = os.path.join(ROOT, "tests", "compile", "gpu_level_forms.cu")
    obj, exe = tmp_path / "gpu_level_forms.o", tmp_path / "gpu_level_forms"
    inc = os.path.join(ROOT, "include")
    r = subprocess.run(f"nvcc -std=c++17 {ARCH} -rdc=true -DCHARMING_GPU_LEVEL -I{inc} -c {src} -o {obj}",
                       shell=True, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run(f"nvcc {ARCH} -rdc=true -Xnvlink -suppress-stack-size-warning -o {exe} {obj} "
                       f"{lib} -lcudart", shell=True, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    # the program defines the symbol the library's process main looks for
    nm = subprocess.run(["nm", "-C", str(exe)], capture_output=True, text=True).stdout
    syms = [l.split() for l in nm.splitlines()]
    assert any(len(f) >= 2 and f[-1] == "charming_program_gpu_level" and f[-2] in ("V", "v", "R")
               for f in syms), nm[-2000:]
