#!/usr/bin/env python
"""Benchmark of the perturbation-MHD hot path on B200.

Headline workload: the 3D gravitationally stratified atmosphere at 512x512x512
mesh cells, the precision-comparison configuration: FP64, RK4
(typeadvance='fourstep'), hyperdiffusion, gravity, bottom velocity driver,
fixed/open x1 boundaries and periodic x2/x3, and an initial state of 64 seeded
random-phase Fourier modes (|k| <= 16, amplitude 1e-4, divergence-free b')
(sac_b200.problems.stratified(perturb=1e-4)).  The stratified-atmosphere
configuration at 128^3, which starts at rest and is stirred by the driver, is
measured beside it.  One step = one time step of the reference's main loop: getdt + advect
(four RK stages with their boundary fills) on the resident state.  Metric:
cell-updates per second (one mesh cell advanced by one full RK4 step), for the
FP64 path and the FP32-perturbation path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 512]

For N>1 the script runs under torch.distributed.run, one process per GPU, each
advancing its own replica (the path does not shard); timing is the max over
ranks, value is the whole-job rate.  `--impl reference` times the CPU
restatement of the reference (oracle/, C++, all host threads) on a bounded
sample of the same workload: the full 128^3 cube (a whole step of the 512^3
grid takes minutes on the host); rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from sac_b200 import abi, problems  # noqa: E402

METRIC = "3D MHD cell-updates/s"
UNIT = "cell-updates/s"
BYTES_PER_CELL_UPDATE = {"fp64": 1056, "fp32": 608}  # 14*n_p*s_p + 4*n_b*s_b, n_p=8, n_b=5
STAGES_PER_STEP = 4
CPU_SAMPLE_N = 128  # the CPU legs time whole RK4 steps of the stratified workload on this cube


MODES_AMP = 1e-4  # the precision-comparison configuration's random-mode amplitude


def perturb_for(n, init):
    """The initial perturbation amplitude of the n^3 workload: the 64 random modes
    of the precision-comparison configuration ('modes'), the state at rest of the
    128^3 configuration ('rest'), or by size ('auto': modes unless n == 128)."""
    if init == "modes" or (init == "auto" and n != 128):
        return MODES_AMP
    return None


def workload(n=128, perturb=None):
    return problems.stratified(n=(n, n, n), perturb=perturb)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(name):
    p = os.path.join(ROOT, "profiles", name)
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        with open(self.file.name) as f:
            rows = [r.split(",") for r in f.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# the CPU legs (oracle = C++ restatement of the reference)
# ---------------------------------------------------------------------------
def cpu_steps(n=CPU_SAMPLE_N, threads=None, seconds=12.0, max_steps=64, min_steps=1, warmup=1, perturb=None):
    """Cell-updates/s of the oracle on the host cores: `warmup` untimed RK4 steps
    (getdt + advect), then timed steps until `seconds` elapse (at least
    min_steps), on the n^3 stratified cube.  Both CPU legs use this."""
    from oracle import oracle

    oracle.build()
    if threads is not None:
        oracle.set_threads(threads)
    P = workload(n, perturb)
    o = oracle.Oracle(P.params)
    o.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    o.set_boundaries(P.typeB_packed, P.nB)
    o.upload(P.w)
    o.getboundary(0.0)
    t, it = 0.0, 0
    for _ in range(warmup):
        dt = o.getdt(it)
        o.advect(dt, t, it)
        t += dt
        it += 1
    k, t0 = 0, time.perf_counter()
    while k < max_steps:
        dt = o.getdt(it)
        o.advect(dt, t, it)
        t += dt
        it += 1
        k += 1
        el = time.perf_counter() - t0
        if k >= min_steps and el > seconds:
            break
    el = time.perf_counter() - t0
    o.close()
    used = threads if threads is not None else oracle.max_threads()
    if threads is not None:
        oracle.set_threads(oracle.max_threads())
    return {"value": P.ncells * k / el, "steps": k, "seconds": el, "threads": used, "cells": P.ncells, "n": n,
            "perturb": perturb}


def cpu_sample_text(r):
    state = "64 random modes, amplitude 1e-4" if r.get("perturb") else "at rest, driven"
    return (f"{r['steps']} RK4 steps (getdt+advect) in {r['seconds']:.1f} s on the full {r['n']}^3 stratified "
            f"cube ({state}), C++ FP64 restatement of the reference (the Fortran reference cannot be built: no Fortran "
            f"compiler), {r['threads']} OpenMP thread(s); a whole RK4 step of the 512^3 grid would take minutes on "
            f"the host, so the cube is the bounded sample of the workload, per cell")


def headline_config(n, world, perturb=None):
    state = ("initial state 64 seeded random modes |k|<=16, amplitude 1e-4, div-free b'" if perturb
             else "initial state at rest")
    return {"workload": f"stratified atmosphere {n}^3, FP64 and FP32-perturbation paths, RK4, hyperdiffusion, "
                        f"gravity, driver, {state}",
            "cells_per_step": n ** 3, "parallelism": f"replicas{world}",
            "l2": f"no flush: the FP64 context holds ~{(n + 4) ** 3 * 800 / 1e9:.1f} GB per replica (state, RK "
                  f"arrays and per-stage intermediates), far larger than the 126 MB L2",
            "step": "getdt + advect (4 RK stages + boundary fills)"}


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    from oracle import oracle

    oracle.build()
    r = cpu_steps(warmup=args.warmup, seconds=0.0, min_steps=args.steps, max_steps=args.steps,
                  perturb=perturb_for(args.n, args.init))
    v = r["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(args.n, world, perturb_for(args.n, args.init)),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["threads"], "kind": "port", "sample": cpu_sample_text(r)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def _lib_ext(ctx):
    lib = ctx.lib
    lib.sac_get_stream.argtypes = [ctypes.c_void_p]
    lib.sac_get_stream.restype = ctypes.c_void_p
    lib.sac_profile.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.sac_profile_read.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_long), ctypes.c_int]
    lib.sac_kernel_launches.argtypes = [ctypes.c_void_p]
    lib.sac_kernel_launches.restype = ctypes.c_long
    return lib


def prof_read(lib, h, kind, reset=True):
    ms, n = ctypes.c_double(), ctypes.c_long()
    lib.sac_profile_read(h, kind, ctypes.byref(ms), ctypes.byref(n), int(reset))
    return ms.value, n.value


KERNELS = ["update", "face", "bound", "courant", "other", "nu"]  # SAC_K_* order


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Max of a per-rank scalar over all ranks (a no-op for one rank).  The tensor
    lives on `device` (the rank's GPU under NCCL, the CPU under gloo)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(cells_per_replica: int, steps: int, world: int, seconds: float) -> float:
    """Whole-job cell-updates/s of `world` replicas that each advanced
    `cells_per_replica` cells by `steps` steps, timed as the slowest rank."""
    return world * cells_per_replica * steps / seconds


def make_ctx(P, local_rank, precision):
    from sac_b200 import params as sp

    P.params.device = local_rank
    P.params.precision = sp.PREC_FP32 if precision == "fp32" else sp.PREC_FP64
    ctx = abi.Context(P.params)
    lib = _lib_ext(ctx)
    ctx.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    ctx.set_boundaries(P.typeB_packed, P.nB)
    ctx.upload(P.w)
    ctx.getboundary(0.0)
    return ctx, lib


def timed_steps(args, P, ctx, lib, local_rank, world, clocks=True):
    """W untimed steps, then K steps between a barrier and CUDA events on the
    library's stream, with per-kernel events and the clock sampler running."""
    import torch
    import torch.distributed as dist

    stream = torch.cuda.ExternalStream(lib.sac_get_stream(ctx.h), device=local_rank)
    t, it = 0.0, 0
    for _ in range(args.warmup):
        dt = ctx.getdt(it)
        ctx.advect(dt, t, it)
        t += dt
        it += 1
    ctx.synchronize()
    lib.sac_profile(ctx.h, 1)
    for k in range(len(KERNELS)):
        prof_read(lib, ctx.h, k, reset=True)
    launches0 = lib.sac_kernel_launches(ctx.h)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank) if clocks else None
    if clk:
        clk.__enter__()
    e0.record(stream)
    for _ in range(args.steps):
        dt = ctx.getdt(it)
        ctx.advect(dt, t, it)
        t += dt
        it += 1
    e1.record(stream)
    torch.cuda.synchronize()
    if clk:
        clk.__exit__()
    ms = e0.elapsed_time(e1)
    if world > 1:
        dist.barrier()
    ms = max_over_ranks(ms, world, device=f"cuda:{local_rank}")
    launches = lib.sac_kernel_launches(ctx.h) - launches0
    kern = {name: prof_read(lib, ctx.h, k) for k, name in enumerate(KERNELS)}
    lib.sac_profile(ctx.h, 0)
    return dict(ms=ms, launches=launches, kern=kern, clocks=clk.summary() if clk else None, t=t, it=it)


SM_COUNT, SCHEDULERS_PER_SM = 148, 4


def issue_ceiling(path, value, sm_mhz, perturb=None):
    """The instruction-issue wall of a path: the warp instructions one RK4 step
    issues per mesh cell (all kernels of the step, ncu instruction counts at 128^3
    from the same initial state, profiles/stage_instructions_stratified128.json)
    against the SM issue peak of one warp instruction per scheduler and clock, at
    the sampled SM clock."""
    p = os.path.join(ROOT, "profiles", "stage_instructions_stratified128.json")
    if not os.path.exists(p) or not sm_mhz:
        return None
    with open(p) as f:
        d = json.load(f)
    key = "warp_instr_per_step_modes" if perturb else "warp_instr_per_step"
    if path not in d.get(key, {}):
        return None
    per_cell = d[key][path] / d["cells"]
    peak = SM_COUNT * SCHEDULERS_PER_SM * sm_mhz * 1e6
    ceiling = peak / per_cell
    return {"warp_instr_per_cell_update": per_cell, "peak_warp_instr_per_s": peak, "unit": "cell-updates/s",
            "ceiling": ceiling, "frac": value / ceiling}


def roofline(b_cell_update, cells, kern, peak, peak_kind, tr_name, label):
    upd_ms, upd_n = kern["update"]
    b_launch = b_cell_update / STAGES_PER_STEP * cells
    achieved = b_launch / (upd_ms / upd_n / 1e3) / 1e9 if upd_n else None
    tr = load_traffic(tr_name)
    traffic = tr["dram_bytes_per_launch"] * cells / tr["cells"] if tr and tr.get("cells") else None
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic, "peak_source": peak_kind,
            "kernel": label, "bytes_per_launch": b_launch, "avg_launch_ms": upd_ms / upd_n if upd_n else None}


def measure(args, n, local_rank, world, legs, clocks=True, perturb=None):
    """The FP64 and FP32 legs (and e2e) of the stratified workload at n^3: each a
    context of its own on the rank's GPU, created, timed and released in turn."""
    import torch
    import torch.distributed as dist

    P = workload(n, perturb)
    cells = P.ncells
    nbytes = P.nw * int(np.prod(P.ixGhi)) * 8
    out = {"cells": cells, "nbytes": nbytes}
    if legs & {"fp64", "e2e"}:
        ctx, lib = make_ctx(P, local_rank, "fp64")
        r64 = timed_steps(args, P, ctx, lib, local_rank, world, clocks=clocks)
        out["r64"] = r64
        out["v64"] = job_rate(cells, args.steps, world, r64["ms"] / 1e3)
        if "e2e" in legs:
            # end to end through the C-ABI with host buffers: per step upload(w),
            # getdt, advect, download(w) from/to pinned host memory
            pin = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
            hw = pin.numpy().reshape(P.ixGhi + (P.nw,), order="F")
            ctx.download(hw)
            t, it = r64["t"], r64["it"]
            e2e_steps = max(3, min(args.steps, 10))
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                ctx.upload(hw)
                dt = ctx.getdt(it)
                ctx.advect(dt, t, it)
                t += dt
                it += 1
                ctx.download(hw)
            e2e_s = max_over_ranks(time.perf_counter() - t0, world, device=f"cuda:{local_rank}")
            out["e2e"] = job_rate(cells, e2e_steps, world, e2e_s)
            del hw, pin
        ctx.close()
        torch.cuda.empty_cache()
    if "fp32" in legs:
        # the FP32-perturbation path on the same workload
        ctx32, lib32 = make_ctx(P, local_rank, "fp32")
        r32 = timed_steps(args, P, ctx32, lib32, local_rank, world, clocks=clocks and "r64" not in out)
        ctx32.close()
        torch.cuda.empty_cache()
        out["r32"] = r32
        out["v32"] = job_rate(cells, args.steps, world, r32["ms"] / 1e3)
    return out


def leg_summary(m, args, peak, peak_kind):
    """Per-path numbers of one workload size for the JSON line."""
    cells = m["cells"]
    d = {"cells_per_step": cells}
    if "r64" in m:
        r = m["r64"]
        d["fp64"] = {"value": m["v64"], "ms_per_step": r["ms"] / args.steps, "gpu_launches": r["launches"],
                     "kernels_ms_per_step": {k: v[0] / args.steps for k, v in r["kern"].items()},
                     "roofline": roofline(BYTES_PER_CELL_UPDATE["fp64"], cells, r["kern"], peak, peak_kind,
                                          "update_fp64_traffic.json",
                                          "k_update<3,3,double> parts A+B (one RK stage)")}
    if "r32" in m:
        r = m["r32"]
        d["fp32"] = {"value": m["v32"], "ms_per_step": r["ms"] / args.steps, "gpu_launches": r["launches"],
                     "speedup_vs_fp64": (m["v32"] / m["v64"]) if "v64" in m else None,
                     "kernels_ms_per_step": {k: v[0] / args.steps for k, v in r["kern"].items()},
                     "roofline": roofline(BYTES_PER_CELL_UPDATE["fp32"], cells, r["kern"], peak, peak_kind,
                                          "update_fp32_traffic.json", "k_update<3,3,float>")}
    return d


def ours(args, rank, world, local_rank):
    import torch

    from sac_b200 import build as sbuild

    sbuild.build()
    torch.cuda.set_device(local_rank)
    legs = set(args.legs.split(","))
    pert = perturb_for(args.n, args.init)
    main = measure(args, args.n, local_rank, world, legs, perturb=pert)
    small = None
    if args.n != 128 and "small" in legs:
        small = measure(args, 128, local_rank, world, legs & {"fp64", "fp32"}, clocks=False,
                        perturb=perturb_for(128, args.init))
    if rank != 0:
        return 0
    peak, peak_kind = load_peaks()
    summ = leg_summary(main, args, peak, peak_kind)
    lead = main.get("r64") or main.get("r32")
    value = main.get("v64", main.get("v32"))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": lead["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if "r64" in main else "f32", "data": "synthetic",
        "config": headline_config(args.n, world, pert),
        "gpu_launches": lead["launches"],
        "clocks": lead["clocks"],
    }
    sm_mhz = (lead["clocks"] or {}).get("sm_mhz")
    if "fp64" in summ:
        line["roofline"] = summ["fp64"]["roofline"]
        line["roofline"]["issue"] = issue_ceiling("fp64", summ["fp64"]["value"] / world, sm_mhz, pert)
        line["kernels_ms_per_step"] = summ["fp64"]["kernels_ms_per_step"]
    if "fp32" in summ:
        summ["fp32"]["roofline"]["issue"] = issue_ceiling("fp32", summ["fp32"]["value"] / world, sm_mhz, pert)
    if "e2e" in main:
        line["e2e"] = {"value": main["e2e"], "unit": UNIT, "h2d_bytes_per_step": main["nbytes"],
                       "d2h_bytes_per_step": main["nbytes"],
                       "path": "sac_upload + sac_getdt + sac_advect + sac_download per step, pinned host w"}
    if "fp32" in summ:
        line["fp32"] = summ["fp32"]
    if small is not None:
        line["stratified_128"] = leg_summary(small, args, peak, peak_kind)
    if world == 1 and not args.no_cpu and "cpu" in legs:
        r = cpu_steps(perturb=pert)
        line["cpu_baseline"] = {"value": r["value"], "unit": UNIT, "cores": r["threads"], "kind": "port",
                                "sample": cpu_sample_text(r)}
        r1 = cpu_steps(n=64, threads=1, seconds=8.0, max_steps=8, perturb=pert)
        line["cpu_baseline_1core"] = {"value": r1["value"], "unit": UNIT, "cores": 1, "kind": "port",
                                      "sample": cpu_sample_text(r1)}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the small configurations' legs (not the headline line): Brio-Wu on the GPU
# through the C-ABI against the CPU oracle, and the CPU oracle on one 2D
# Orszag-Tang instance of the batch's mean size (the batch's CPU baseline)
# ---------------------------------------------------------------------------
def _start(cls, P):
    c = cls(P.params)
    c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    c.set_boundaries(P.typeB_packed, P.nB)
    c.upload(P.w)
    c.getboundary(0.0)
    return c


def _to_tmax(c, tmax, max_steps=100000):
    """program vac's loop (getdt, then advect) until t reaches tmax."""
    t, it = 0.0, 0
    while t < tmax and it < max_steps:
        dt = min(c.getdt(it), tmax - t + 1e-99)
        c.advect(dt, t, it)
        t += dt
        it += 1
    return it


def briowu_workload():
    """Brio-Wu (1D, nx=800, to t=0.1): the GPU through the C-ABI, each getdt
    reading its reductions back, with CUDA events around the loop; the CPU
    oracle on all host threads and on one; the GPU's relative L2 to the oracle."""
    import ctypes

    import torch

    from oracle import oracle

    from sac_b200 import abi, build, problems
    build.build()
    oracle.build()
    nthreads = oracle.max_threads()
    P = problems.brio_wu()
    out = {"workload": "Brio-Wu 1D nx=800 to t=0.1, FP64, RK4, hyperdiffusion, Courant 0.8"}
    g = _start(abi.Context, P)
    g.lib.sac_get_stream.argtypes = [ctypes.c_void_p]
    g.lib.sac_get_stream.restype = ctypes.c_void_p
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
    out["gpu"] = {"steps": n, "ms": ms, "cell_updates_per_s": P.ncells * n / (ms / 1e3)}
    for threads in (nthreads, 1):
        oracle.set_threads(threads)
        o = _start(oracle.Oracle, P)
        t0 = time.perf_counter()
        n2 = _to_tmax(o, P.tmax)
        el = time.perf_counter() - t0
        wo = o.download()
        o.close()
        out[f"cpu_{threads}_threads"] = {"steps": n2, "s": el, "cell_updates_per_s": P.ncells * n2 / el}
    oracle.set_threads(nthreads)
    out["gpu_vs_oracle_rel_l2"] = float(np.linalg.norm((wg - wo)[2:-2, :6]) / np.linalg.norm(wo[2:-2, :6]))
    return out


def batch_cpu_workload(steps=5):
    """The CPU oracle on one 288 x 288 Orszag-Tang instance (the batch's mean size)
    on all host threads: one untimed step, then `steps` timed ones."""
    from oracle import oracle

    from sac_b200 import problems
    oracle.build()
    nthreads = oracle.max_threads()
    Q = problems.orszag_tang((288, 288), beta=2.0)
    o = _start(oracle.Oracle, Q)
    t = 0.0
    for it in range(steps + 1):
        if it == 1:
            t0 = time.perf_counter()
        dt = o.getdt(it)
        o.advect(dt, t, it)
        t += dt
    el = time.perf_counter() - t0
    o.close()
    return {"workload": "one Orszag-Tang instance 288 x 288, FP64, RK4, hyperdiffusion (CPU oracle)",
            "steps": steps, "s": el, "cell_updates_per_s": Q.ncells * steps / el, "threads": nthreads}


def batch_workload(args):
    """The batched configuration: 4096 uneven Orszag-Tang vortices (nx, ny from
    {64, 96, ..., 512}), every instance with its own dt, FP64 and FP32, each a
    CUDA-graph replay per RK4 step (sac_b200.batch_bench)."""
    import torch

    from sac_b200 import batch_bench, build, params

    build.build()
    torch.cuda.init()
    out = {"workload": "4096 uneven Orszag-Tang vortices, RK4, hyperdiffusion, own dt per instance"}
    for name, prec in (("fp64", params.PREC_FP64), ("fp32", params.PREC_FP32)):
        out[name] = batch_bench.run(4096, max(args.steps, 3), max(args.warmup, 1), prec)
        torch.cuda.empty_cache()
    out["fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


def smallfix_workload(args):
    """keeppositive on the device: the Orszag-Tang vortex at 512^2 with the floors
    of its initial state (smallp 0.5, smallrho = vacuumrho = 2.75), FP64, RK4 with
    hyperdiffusion, K steps after W untimed ones (each fill runs keeppositive)."""
    from sac_b200 import build

    build.build()
    P = problems.orszag_tang((512, 512))
    P.params.smallfix = 1
    P.params.smallp = 0.5
    P.params.smallrho = 2.75
    P.params.vacuumrho = 2.75
    c = abi.Context(P.params)
    c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    c.set_boundaries(P.typeB_packed, P.nB)
    c.upload(P.w)
    c.getboundary(0.0)
    t, it = 0.0, 0
    for _ in range(max(args.warmup, 1)):
        dt = c.getdt(it)
        c.advect(dt, t, it)
        t, it = t + dt, it + 1
    c.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dt = c.getdt(it)
        c.advect(dt, t, it)
        t, it = t + dt, it + 1
    c.synchronize()
    el = time.perf_counter() - t0
    d = c.diag()
    c.close()
    return {"workload": "Orszag-Tang 512^2 with keeppositive floors, FP64, RK4, hyperdiffusion",
            "steps": args.steps, "s": el, "cell_updates_per_s": P.ncells * args.steps / el,
            "nerror_toosmallp": d.nerror_toosmallp}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512, help="mesh cells per dimension of the headline line (default 512)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--init", default="auto", choices=["auto", "modes", "rest"],
                    help="initial state: the 64 random modes of the precision-comparison configuration, the state "
                         "at rest of the 128^3 configuration, or auto (modes unless --n 128)")
    ap.add_argument("--legs", default="fp64,e2e,fp32,small,cpu",
                    help="comma list of fp64, e2e, fp32, small (the 128^3 legs beside a larger --n), cpu "
                         "(profiling runs select one kernel family)")
    ap.add_argument("--workload", default="stratified",
                    choices=["stratified", "briowu", "batch", "batch-cpu", "smallfix"],
                    help="stratified: the headline line; briowu / batch / batch-cpu: the other configurations' legs; "
                         "smallfix: keeppositive on a 2D vortex (profiling)")
    args = ap.parse_args()
    if args.workload != "stratified":
        res = {"briowu": briowu_workload, "batch-cpu": batch_cpu_workload,
               "batch": lambda: batch_workload(args), "smallfix": lambda: smallfix_workload(args)}[args.workload]()
        print(json.dumps(res), flush=True)
        return 0
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
