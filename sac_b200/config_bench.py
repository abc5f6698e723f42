"""Time the small workloads that bench.py does not: Brio-Wu (1D, nx=800, to
t=0.1) on the GPU and on the CPU oracle, and the CPU oracle on one 2D
Orszag-Tang instance of the batch's mean size (the CPU baseline of the batch).

    python -m sac_b200.config_bench

Prints one JSON line.  The GPU leg runs the reference's main loop through the
C-ABI (getdt + advect per step, each getdt reading its reductions back), with
CUDA events around the loop; the CPU legs use the oracle (OpenMP on all host
threads, and one thread).
"""
from __future__ import annotations

import json
import time

import numpy as np

from . import abi, problems


def _start(cls, P, **kw):
    c = cls(P.params, **kw) if kw else cls(P.params)
    c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    c.set_boundaries(P.typeB_packed, P.nB)
    c.upload(P.w)
    c.getboundary(0.0)
    return c


def _to_tmax(c, tmax, max_steps=100000):
    t, it = 0.0, 0
    while t < tmax and it < max_steps:
        dt = min(c.getdt(it), tmax - t + 1e-99)
        c.advect(dt, t, it)
        t += dt
        it += 1
    return it


def _steps(c, n):
    t = 0.0
    for it in range(n):
        dt = c.getdt(it)
        c.advect(dt, t, it)
        t += dt


def main(argv=None):
    import torch

    from oracle import oracle

    from . import build
    build.build()
    oracle.build()
    nthreads = oracle.max_threads()
    out = {}
    # Brio-Wu on the GPU
    P = problems.brio_wu()
    g = _start(abi.Context, P)
    g.lib.sac_get_stream.argtypes = [abi.ctypes.c_void_p]
    g.lib.sac_get_stream.restype = abi.ctypes.c_void_p
    st = torch.cuda.ExternalStream(g.lib.sac_get_stream(g.h))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    n = _to_tmax(g, P.tmax)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    wg = g.download()
    g.close()
    out["briowu_gpu"] = {"steps": n, "ms": ms, "cell_updates_per_s": P.ncells * n / (ms / 1e3)}
    # Brio-Wu on the CPU oracle, all threads and one
    for threads in (nthreads, 1):
        oracle.set_threads(threads)
        o = _start(oracle.Oracle, P)
        t0 = time.perf_counter()
        n2 = _to_tmax(o, P.tmax)
        el = time.perf_counter() - t0
        wo = o.download()
        o.close()
        out[f"briowu_cpu_{threads}t"] = {"steps": n2, "s": el, "cell_updates_per_s": P.ncells * n2 / el}
    err = np.linalg.norm((wg - wo)[2:-2, :6]) / np.linalg.norm(wo[2:-2, :6])
    out["briowu_gpu_vs_oracle_rel_l2"] = float(err)
    # one 288 x 288 Orszag-Tang instance on the CPU oracle (the batch's mean size)
    oracle.set_threads(nthreads)
    Q = problems.orszag_tang((288, 288), beta=2.0)
    o = _start(oracle.Oracle, Q)
    _steps(o, 1)
    t0 = time.perf_counter()
    k = 5
    _steps(o, k)
    el = time.perf_counter() - t0
    o.close()
    out["ot288_cpu"] = {"steps": k, "s": el, "cell_updates_per_s": Q.ncells * k / el,
                        "threads": nthreads}
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
