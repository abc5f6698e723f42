"""FP32-perturbation path against the plain FP64 path on the same GPU.

    python -m sac_b200.precision --n 512 --steps 1000 [--out result.json]

Workload: the stratified atmosphere at n^3 with a seeded perturbation of 64
random-phase Fourier modes, |k| <= 16, amplitude 1e-4, divergence-free b'
(sac_b200.problems.stratified(perturb=1e-4)).  The FP64 context advances the
state with its own getdt; the FP32 context then advances the same initial state
with the FP64 run's dt sequence, so that the comparison measures the storage
precision of the perturbations and not the dt noise of the hyperdiffusion
coefficient.  Both runs are timed on the device (CUDA events on the library
stream), getdt included.  Reported per advanced variable: relative L2 and L-inf
(relative to the FP64 field's max) over the mesh, and the 4th-order div b of
both runs (sac_diag).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import abi, params, problems


def _ctx(P, precision):
    P.params.precision = precision
    c = abi.Context(P.params)
    c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    c.set_boundaries(P.typeB_packed, P.nB)
    c.upload(P.w)
    c.getboundary(0.0)
    return c


def _run(c, steps, dts=None, log=print):
    import torch
    lib = c.lib
    lib.sac_get_stream.argtypes = [abi.ctypes.c_void_p]
    lib.sac_get_stream.restype = abi.ctypes.c_void_p
    st = torch.cuda.ExternalStream(lib.sac_get_stream(c.h))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    used = []
    t = 0.0
    torch.cuda.synchronize()
    e0.record(st)
    for k in range(steps):
        d = c.getdt(k)
        if dts is not None:
            d = dts[k]
        c.advect(d, t, k)
        t += d
        used.append(d)
        if k % 100 == 99:
            log(f"  step {k + 1}/{steps}")
    e1.record(st)
    e1.synchronize()
    return used, e0.elapsed_time(e1)


def compare(w64, w32, P):
    sl = tuple(slice(2, 2 + n) for n in P.nx)
    names = ["rho"] + [f"m{c + 1}" for c in range(P.ndir)] + ["e"] + [f"b{c + 1}" for c in range(P.ndir)]
    out = {}
    for iw, nm in enumerate(names):
        a = w64[sl + (iw,)]
        b = w32[sl + (iw,)]
        d = b - a
        na = float(np.sqrt(np.sum(a * a)))
        out[nm] = {"rel_l2": float(np.sqrt(np.sum(d * d))) / max(na, 1e-300),
                   "rel_linf": float(np.abs(d).max()) / max(float(np.abs(a).max()), 1e-300)}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--amp", type=float, default=1e-4)
    ap.add_argument("--out", default=None)
    ap.add_argument("--twin-eps", type=float, default=0.0,
                    help="also run an FP64 twin whose rho' differs by this relative amount")
    a = ap.parse_args(argv)
    import torch
    torch.cuda.init()
    from . import build
    build.build()
    log = lambda m: print(m, flush=True)  # noqa: E731
    t0 = time.time()
    P = problems.stratified(n=(a.n,) * 3, perturb=a.amp)
    log(f"initial state {a.n}^3 built in {time.time() - t0:.1f} s")
    cells = P.ncells
    c64 = _ctx(P, params.PREC_FP64)
    dts, ms64 = _run(c64, a.steps, log=log)
    d64 = c64.diag()
    w64 = c64.download()
    c64.close()
    torch.cuda.empty_cache()
    log(f"FP64: {a.steps} steps in {ms64 / 1e3:.1f} s")
    c32 = _ctx(P, params.PREC_FP32)
    _, ms32 = _run(c32, a.steps, dts=dts, log=log)
    d32 = c32.diag()
    w32 = c32.download()
    c32.close()
    log(f"FP32: {a.steps} steps in {ms32 / 1e3:.1f} s")
    errs = compare(w64, w32, P)
    twin = None
    if a.twin_eps > 0:
        # the same FP64 run from an initial rho' perturbed at the eps level
        rng = np.random.default_rng(11)
        rho = P.w[..., 0]
        P.w[..., 0] = rho + a.twin_eps * np.abs(rho).max() * rng.uniform(-1, 1, rho.shape)
        ct = _ctx(P, params.PREC_FP64)
        _run(ct, a.steps, dts=dts, log=log)
        wt = ct.download()
        ct.close()
        tw = compare(w64, wt, P)
        twin = {"eps": a.twin_eps, "max_rel_l2": max(v["rel_l2"] for v in tw.values()), "per_variable": tw}
    res = {"workload": f"stratified {a.n}^3, 64 random modes |k|<=16 amplitude {a.amp}, div-free b'",
           "steps": a.steps, "cells": cells, "t_end": float(sum(dts)),
           "fp64_cell_updates_per_s": cells * a.steps / (ms64 / 1e3),
           "fp32_cell_updates_per_s": cells * a.steps / (ms32 / 1e3),
           "fp32_over_fp64": ms64 / ms32,
           "max_rel_l2": max(v["rel_l2"] for v in errs.values()), "per_variable": errs,
           "divb_l2": {"fp64": d64.divb_l2, "fp32": d32.divb_l2},
           "divb_linf": {"fp64": d64.divb_linf, "fp32": d32.divb_linf},
           "dt_first_last": [dts[0], dts[-1]], "fp64_twin": twin}
    log(json.dumps(res))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    return res


if __name__ == "__main__":
    main()
