"""Build libsacgpu.so (sm_100a) in-tree with nvcc.

The library is compiled with --fmad=false: every a*b+c in the FP64 stage is
rounded twice, as the reference's Fortran expressions are evaluated, so that the
device results agree with the CPU oracle to rounding.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsacgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if p and os.path.exists(p):
            return p
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh", ".h"))]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = sources() + [os.path.join(ROOT, "include", "sac_gpu.h"), __file__]
    return all(os.path.getmtime(s) <= t for s in deps)


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return OUT
    cmd = [nvcc_path(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
           "-shared", "-I", os.path.join(ROOT, "include"), "-o", OUT + ".tmp",
           os.path.join(CSRC, "sac_gpu.cu"), *extra]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(OUT)
