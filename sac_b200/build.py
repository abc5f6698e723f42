"""Build the in-tree sm_100a libraries with nvcc.

libsacgpu.so   the perturbation-MHD path (single grid and batch), csrc/
libsacfno.so   the Fourier-neural-operator surrogate, csrc/fno/

The solver's host unit and FP64 stage keep every rounding of the reference (no
FMA contraction, IEEE division and square root); the FP32 stage may contract and
approximate.  The surrogate computes in BF16 with FP32 accumulation.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsacgpu.so")
FNO_OUT = os.path.join(HERE, "libsacfno.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# library -> (source dir, [(translation unit, flags)], public header)
LIBS = {
    OUT: (CSRC, [
        ("sac_gpu.cu", ["--fmad=false"]),
        ("stage_f64.cu", ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
        ("stage_f32.cu", ["--fmad=true", "-prec-div=false", "-ftz=true"]),
        ("sac_batch.cu", ["--fmad=false"]),
        ("stage_joint.cu", ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ], "sac_gpu.h"),
    FNO_OUT: (os.path.join(CSRC, "fno"), [
        ("fno_gemm.cu", []),
        ("fno_net.cu", []),
    ], "sac_fno.h"),
}
UNITS = LIBS[OUT][1]


def nvcc_path():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if p and os.path.exists(p):
            return p
    raise RuntimeError("nvcc not found")


def _sources(d):
    return [os.path.join(d, f) for f in sorted(os.listdir(d)) if f.endswith((".cu", ".cuh", ".h"))]


def up_to_date(out=OUT):
    if not os.path.exists(out):
        return False
    src, _, header = LIBS[out]
    t = os.path.getmtime(out)
    deps = _sources(src) + [os.path.join(ROOT, "include", header), __file__]
    return all(os.path.getmtime(s) <= t for s in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)


def _build_lib(out, force=False, verbose=False, extra=()):
    if not force and up_to_date(out):
        return out
    src, units, _ = LIBS[out]
    objdir = os.path.join(HERE, "_build", os.path.basename(out).replace(".so", ""))
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for unit, flags in units:
        obj = os.path.join(objdir, unit.replace(".cu", ".o"))
        cmds.append([nvcc_path(), "-O3", "-std=c++17", *ARCH, "-lineinfo", *flags, "-Xcompiler", "-fPIC",
                     "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-c", "-o", obj, os.path.join(src, unit),
                     *extra])
        objs.append(obj)
    # the translation units compile independently: one nvcc each, side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, c, verbose) for c in cmds]:
            f.result()
    _run([nvcc_path(), *ARCH, "-shared", "-o", out + ".tmp", *objs], verbose)
    os.replace(out + ".tmp", out)
    return out


def build(force=False, verbose=False, extra=()):
    """libsacgpu.so (the solver); returns its path."""
    return _build_lib(OUT, force, verbose, extra)


def build_fno(force=False, verbose=False, extra=()):
    """libsacfno.so (the surrogate); returns its path."""
    return _build_lib(FNO_OUT, force, verbose, extra)


if __name__ == "__main__":
    ex = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    f = "--force" in sys.argv
    if "--fno" not in sys.argv or "--all" in sys.argv:
        print(build(force=f, verbose=True, extra=ex))
    if "--fno" in sys.argv or "--all" in sys.argv:
        print(build_fno(force=f, verbose=True, extra=ex))
