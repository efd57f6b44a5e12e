"""The device API forms of the reference's headers compile against include/
and link against libcharming.a (nvcc cross-compiles for sm_100a without a
GPU): the const message invoke overloads, malloc_user / free_user and
async_wait (tests/compile/api_forms.cu)."""
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
