"""Build program vac with its hot path on the GPU: the reference's Fortran host
(drewleonard42/SAC src/*.t) calling libsacgpu.so through include/sac_gpu_mod.f90.

    python -m sac_b200.fortran.host_build --ref <SAC>/src --out <build dir> [--fc gfortran]

The steps follow the reference's own build driver (sac/src/sac_fabricate.py:
preprocess every .t with vacpp.sh, compile the vacdef module first, then the
sources, then link) with three differences:
  - the interface module include/sac_gpu_mod.f90 is compiled before vacdef;
  - a copy of src/vac.t is rewritten (patch_vac below) so that its call sites call
    the GPU routines of vacgpu.t, which is preprocessed and compiled with the rest;
  - the link adds libsacgpu.so and the CUDA runtime.
The reference tree is only read: everything is written under --out.  A Fortran
compiler is required; without one the build stops with a message saying so.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
MODULE = os.path.join(ROOT, "include", "sac_gpu_mod.f90")
SHIM = os.path.join(HERE, "vacgpu.t")

SOURCES = ["vac", "vacio", "vacgrid", "vacphys0", "vacphys", "vacusr", "vaccd", "vacgpu"]
INCLUDES = ["vacusrpar", "vacpar"]
MODULES = ["vacdef"]

# The call sites of program vac and advance_expl that move to the GPU, as the
# reference's src/vac.t writes them (stripped of leading blanks), each with its
# replacement.  Every pattern must occur exactly as often as stated, so that a
# changed reference is detected instead of half-patched.
PATCHES = [
    # the first ghost fill after startup (src/vac.t:54, at the start of its line,
    # unlike the split-source fills): the device takes over
    ("\ncall getboundary(t,1,nw,1,ndim,w)\n", "\ncall gpuini(w)\n", 1),
    # the saves of the main loop and of the end (src/vac.t:57,112)
    ("if(timetosave(ifile)) call savefile(ifile,w)",
     "if(timetosave(ifile))then\ncall gpudownload(w)\ncall savefile(ifile,w)\nendif", 1),
    ("if(itsavelast(ifile)<it)call savefile(ifile,w)",
     "if(itsavelast(ifile)<it)then\ncall gpudownload(w)\ncall savefile(ifile,w)\nendif", 1),
    # advect in advance_expl (src/vac.t:317,323,329)
    ("call advect(method,ix^L,iws,idimsplit,idimsplit,w1,w)", "call gpuadvect(method,iws,idimsplit,idimsplit)", 2),
    ("call advect(method,ix^L,iws,1,ndim,w1,w)", "call gpuadvect(method,iws,1,ndim)", 1),
    # the residual needs the advanced state on the host (src/vac.t:90)
    ("if(residmin>zero .or. residmax<bigdouble)then\n      ! calculate true residual",
     "if(residmin>zero .or. residmax<bigdouble)then\ncall gpudownload(w)\n      ! calculate true residual", 1),
]
# the dt block (src/vac.t:61-70): everything from `if(dtpar>zero)then` to its
# `endif` becomes one call; dtmrpc, slowsteps and tmaxexact stay on the host
DT_BLOCK_START = "if(dtpar>zero)then"
DT_BLOCK_LINES = ["dt=dtpar", "else", "if(courantpar>zero)call getdt_courant(w,ixM^L)", "call getdt(w,ixM^L)",
                  "call getdt_special(w,ixM^L)", "", "if(dtcantgrow.and.it>itmin)dt=min(dt,dtold)", "dtold=dt",
                  "endif"]


class PatchError(RuntimeError):
    pass


def patch_vac(text: str) -> str:
    """src/vac.t with its hot-path call sites replaced by the GPU routines."""
    lines = text.split("\n")
    # the dt block
    starts = [i for i, ln in enumerate(lines) if ln.strip() == DT_BLOCK_START]
    if len(starts) != 1:
        raise PatchError(f"the dt block start occurs {len(starts)} times")
    i0 = starts[0]
    k = i0 + 1
    for want in DT_BLOCK_LINES:
        while want and k < len(lines) and not lines[k].strip():
            k += 1
        if want and (k >= len(lines) or lines[k].strip() != want):
            raise PatchError(f"dt block: expected '{want}' at line {k + 1}")
        if want:
            k += 1
    lines[i0:k] = ["   call gpugetdt(w)"]
    out = "\n".join(lines)
    for pat, rep, count in PATCHES:
        n = out.count(pat)
        if n != count:
            raise PatchError(f"'{pat.strip().splitlines()[0]}' occurs {n} times, expected {count}")
        out = out.replace(pat, rep)
    # release the device context before the end-of-run report
    fin = "if(verbose)write(*,'(a,f10.3,a)')'Finish Advance ',time1,' sec'"
    if out.count(fin) != 1:
        raise PatchError("the 'Finish Advance' report occurs other than once")
    out = out.replace(fin, "call gpufinish\n" + fin)
    return out


def fortran_compiler(fc=None):
    for c in (fc, os.environ.get("FC"), "gfortran", "ifort", "ifx", "flang", "mpif90"):
        if c and shutil.which(c):
            return shutil.which(c)
    return None


def _run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed:\n{r.stdout}\n{r.stderr}")


def build(ref_src: str, out: str, fc=None, flags=("-ffree-form", "-ffree-line-length-none", "-O2"),
          cuda_lib="/usr/local/cuda/lib64") -> str:
    """Preprocess, patch, compile and link; returns the path of the vac binary."""
    comp = fortran_compiler(fc)
    if comp is None:
        raise RuntimeError("no Fortran compiler found (gfortran, ifort, ifx, flang, mpif90): "
                           "the host cannot be built on this machine")
    from sac_b200 import build as sbuild

    lib = sbuild.build()
    os.makedirs(out, exist_ok=True)
    for name in os.listdir(ref_src):
        if name.endswith(".t") or name in ("vacpp.pl", "vacpp.sh") or name.startswith("vacusr") \
                or name.startswith("vacpar") or name.startswith("vacphys"):
            shutil.copy(os.path.join(ref_src, name), os.path.join(out, name))
    with open(os.path.join(out, "vac.t")) as f:
        patched = patch_vac(f.read())
    with open(os.path.join(out, "vac.t"), "w") as f:
        f.write(patched)
    shutil.copy(SHIM, os.path.join(out, "vacgpu.t"))
    pre = "./vacpp.sh" if os.path.exists(os.path.join(out, "vacpp.sh")) else None
    for src in SOURCES + MODULES + INCLUDES:
        if pre:
            _run(["sh", pre, src + ".t", src + ".f90"], out)
        else:
            with open(os.path.join(out, src + ".f90"), "w") as f:
                subprocess.run(["perl", "vacpp.pl", src + ".t"], cwd=out, stdout=f, check=True)
    _run([comp, *flags, "-c", MODULE], out)
    for src in MODULES:
        _run([comp, *flags, "-c", src + ".f90"], out)
    for src in SOURCES:
        _run([comp, *flags, "-c", src + ".f90"], out)
    exe = os.path.join(out, "vac")
    _run([comp, "-o", exe, *[s + ".o" for s in SOURCES + MODULES], "sac_gpu_mod.o",
          "-L" + os.path.dirname(lib), "-lsacgpu", "-L" + cuda_lib, "-lcudart",
          "-Wl,-rpath," + os.path.dirname(lib)], out)
    return exe


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's src directory (read only)")
    ap.add_argument("--out", required=True, help="build directory")
    ap.add_argument("--fc", default=None, help="Fortran compiler")
    a = ap.parse_args(argv)
    try:
        print(build(a.ref, a.out, a.fc))
    except RuntimeError as e:
        print(str(e), file=sys.stderr)
        return 2
    return 0


if __name__ == "__main__":
    sys.exit(main())
