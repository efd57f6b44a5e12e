"""Build recipe: the sm_100a runtime (charming_b200/lib), the CPU oracle
(oracle/liboracle_jacobi.so), and, when the reference tree is present, the
reference's examples linked unchanged against libcharming.a
(build/ref_examples/) and the reference-kernel harness (oracle/_ref/)."""
from __future__ import annotations

import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "charming_b200", "csrc")
# The reference tree (only where it is present): CHARMING_REFERENCE, else a
# directory named "reference" beside this repository.
REFERENCE = os.environ.get("CHARMING_REFERENCE",
                           os.path.join(os.path.dirname(ROOT), "reference"))
ARCH = "-gencode arch=compute_100a,code=sm_100a"
REF_EXAMPLES = ("hello", "refnum", "pingpong")
REF_EXAMPLES_GPU_LEVEL = ("pingpong",)
# the multi-GPU build of the library (several GPUs, or virtual GPUs on one)
MULTI = "VARIANT=_multi EXTRA_NVFLAGS=-DCHARMING_MULTI_GPU"


def _run(cmd: str, cwd: str) -> None:
    r = subprocess.run(cmd, cwd=cwd, shell=True, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout[-4000:] + r.stderr[-4000:])
        raise RuntimeError(f"build step failed ({cwd}): {cmd}")


def build_runtime(jobs: int = 8) -> None:
    _run(f"make -j{jobs}", CSRC)
    # the same runtime with invariant checks (CHARMING_CHECKED=1 selects it)
    _run(f"make -j{jobs} CHECKS=1", CSRC)
    _run(f"make -j{jobs} {MULTI}", CSRC)


def build_oracle() -> None:
    _run("make", os.path.join(ROOT, "oracle"))


def build_reference_artifacts() -> bool:
    """Reference examples against this runtime, and the reference-kernel
    harness. Only where the reference tree exists (the build container)."""
    if not os.path.isdir(os.path.join(REFERENCE, "examples")):
        return False
    out = os.path.join(ROOT, "build", "ref_examples")
    os.makedirs(out, exist_ok=True)
    lib = os.path.join(ROOT, "charming_b200", "lib", "libcharming.a")
    inc = os.path.join(ROOT, "include")
    # SM-level builds of every example, and GPU-level builds (the examples'
    # #ifndef SM_LEVEL branch, the reference's default) of those that have one
    lib_multi = os.path.join(ROOT, "charming_b200", "lib", "libcharming_multi.a")
    builds = [(ex, ex, "", lib) for ex in REF_EXAMPLES]
    builds += [(ex, f"{ex}_gpu_level", "-DCHARMING_GPU_LEVEL", lib) for ex in REF_EXAMPLES_GPU_LEVEL]
    # against the multi-GPU build: several GPUs (WORLD_SIZE, or CHARMING_VIRTUAL_DEVS)
    builds += [(ex, f"{ex}_multi", "", lib_multi) for ex in REF_EXAMPLES]
    for ex, name, flags, lib in builds:
        src = os.path.join(REFERENCE, "examples", ex, f"{ex}.cu")
        obj = os.path.join(out, f"{name}.o")
        _run(f"nvcc -std=c++17 -O2 {ARCH} -rdc=true {flags} -I{inc} -I{os.path.dirname(src)} "
             f"-c {src} -o {obj}", ROOT)
        _run(f"nvcc {ARCH} -rdc=true -Xnvlink -suppress-stack-size-warning "
             f"-o {os.path.join(out, name)} {obj} {lib} -lcudart", ROOT)
    _run(f"make REF={REFERENCE}", os.path.join(ROOT, "oracle", "ref"))
    return True


def build_all() -> None:
    build_runtime()
    build_oracle()
    build_reference_artifacts()


if __name__ == "__main__":
    build_all()
