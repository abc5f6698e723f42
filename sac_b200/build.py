"""Build libsacgpu.so (sm_100a) in-tree with nvcc.

Floating-point contraction (FMA) is on; the parity bar against the CPU oracle
(1e-12 relative L2 in FP64) leaves room for the one-rounding differences it makes.
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


# translation units and their floating-point flags: the host file and the FP64
# stage keep every rounding of the reference (no FMA contraction, IEEE division);
# the FP32 stage may contract and approximate.
UNITS = [
    ("sac_gpu.cu", ["--fmad=false"]),
    ("stage_f64.cu", ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("stage_f32.cu", ["--fmad=true", "-prec-div=false", "-ftz=true"]),
    ("sac_batch.cu", ["--fmad=false"]),
]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src, flags in UNITS:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        _run([nvcc_path(), "-O3", "-std=c++17", *ARCH, "-lineinfo", *flags, "-Xcompiler", "-fPIC",
              "-I", os.path.join(ROOT, "include"), "-c", "-o", obj, os.path.join(CSRC, src), *extra], verbose)
        objs.append(obj)
    _run([nvcc_path(), *ARCH, "-shared", "-o", OUT + ".tmp", *objs], verbose)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(OUT)
