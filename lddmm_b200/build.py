"""Build the sm_100a shared library in-tree: lddmm_b200/liblddmm_b200.so.

    python -m lddmm_b200.build            # or: python lddmm_b200/build.py

One nvcc invocation over lddmm_b200/csrc/lddmm_b200.cu (which includes the kernel
headers) and lddmm_b200/csrc/warmstart.cu (the warm-start network), static CUDA runtime, no fast-math (the approximate MUFU instructions
used in the pair loops are written explicitly; everything else keeps IEEE FP32/FP64).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "liblddmm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".h"))] + [
        os.path.join(os.path.dirname(HERE), "include", "lddmm_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-cudart", "static", "-Xptxas", "-v" if verbose else "-O3",
           "-I", os.path.join(os.path.dirname(HERE), "include"),
           os.path.join(CSRC, "lddmm_b200.cu"), os.path.join(CSRC, "warmstart.cu"),
           "-o", OUT + ".tmp"]
    if extra:
        cmd[1:1] = list(extra)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
