"""Throughput of the batched path on uneven Orszag-Tang vortices.

    python -m sac_b200.batch_bench --ninst 4096 --steps 10 --warmup 3 --precision both
    python -m sac_b200.batch_bench --ninst 2048 --steps 10 --warmup 3 --joint

Builds the batch (sizes nx, ny drawn from {64, 96, ..., 512}, beta uniform in
[0.5, 10], seeded), lets the autotuner pick the update tile, replays the
captured RK4 step W times untimed, then times K steps with CUDA events on the
batch's stream.  Prints one JSON line per precision: mesh cell-updates/s over
the whole batch (every instance advances one step per replay, each with its own
dt), ms per step, the tile chosen, the device memory the batch holds and the
spread of the instances' simulated times.

--joint builds the same instances in FP64 and in FP32, tunes each, times them
advanced separately (each batch's own graph on its own stream, both per step),
then joins them (sac_batch_join) and times the joined step in both join forms
(joint kernels, where every kernel covers the tiles of both batches in one
launch, and two graph branches); `value` is the form the join chose.
"""
from __future__ import annotations

import argparse
import json
import time


from . import batch, params


def run(ninst, steps, warmup, precision, seed=0, group_cells=0, tune=True, sizes=batch.OT_SIZES,
        verbose=False, stage=None):
    import torch

    gen = batch.OTBatch(ninst, seed=seed, sizes=sizes)
    prm = batch.ot_params(precision=precision)
    t0 = time.time()
    free0 = torch.cuda.mem_get_info()[0]
    b = gen.make(prm, group_cells=group_cells)
    setup_s = time.time() - t0
    held = free0 - torch.cuda.mem_get_info()[0]
    tile, tune_ms = b.tune() if tune else ((32, 8), 0.0)
    if stage is not None:
        b.set_stage(*stage)
    fused, shape, ms3, msf = b.stage()
    stream = torch.cuda.ExternalStream(b.stream())
    b.advance(warmup)
    b.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.advance(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    t, dt, it = b.state()
    cells = b.mesh_cells
    out = {
        "metric": "batched 2D MHD mesh cell-updates/s",
        "value": cells * steps / (ms / 1e3),
        "unit": "cell-updates/s",
        "precision": "fp32" if precision == params.PREC_FP32 else "fp64",
        "ninst": ninst,
        "mesh_cells": cells,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": ms / steps,
        "tile": list(tile),
        "tune_update_ms": tune_ms,
        "stage": {"fused": fused, "fused_tile": [[32, 8], [16, 8]][shape], "tune_ms_three_pass": ms3,
                  "tune_ms_fused": msf},
        "device_bytes": int(held),
        "setup_s": setup_s,
        "t_min": float(t.min()), "t_max": float(t.max()),
        "dt_min": float(dt.min()), "dt_max": float(dt.max()),
        "steps_done": int(it.min()),
        "config": {"workload": "uneven Orszag-Tang batch", "sizes": f"{sizes[0]}..{sizes[-1]} step "
                   f"{sizes[1] - sizes[0]}", "beta": "U[0.5,10]", "seed": seed, "group_cells": group_cells},
    }
    b.close()
    return out


def _timed(b, steps, warmup, others=()):
    """ms of `steps` replays of b's step (and of each batch in others, on its own
    stream), CUDA events on b's stream after `warmup` untimed ones; the end event
    follows a host wait for the others."""
    import torch

    stream = torch.cuda.ExternalStream(b.stream())
    for x in (b,) + tuple(others):
        x.synchronize()
    for _ in range(warmup):
        b.advance(1)
        for x in others:
            x.advance(1)
    for x in (b,) + tuple(others):
        x.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        b.advance(1)
        for x in others:
            x.advance(1)
    for x in others:
        x.synchronize()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_joint(ninst, steps, warmup, seed=0, sizes=batch.OT_SIZES):
    gen = batch.OTBatch(ninst, seed=seed, sizes=sizes)
    b64 = gen.make(batch.ot_params(precision=params.PREC_FP64))
    b32 = gen.make(batch.ot_params(precision=params.PREC_FP32))
    b64.tune()
    b32.tune()
    b32.set_stage(True, b64.stage()[1])  # the join runs both in the lead's tile shape
    b64.set_stage(True, b64.stage()[1])
    cells = b64.mesh_cells + b32.mesh_cells
    ms_seq = _timed(b64, steps, warmup, others=(b32,))
    b64.join(b32)
    form, stage_joint, stage_forked = b64.join_info()
    ms_form = {}
    for f in (0, 1):
        b64.set_join_form(f)
        ms_form[f] = _timed(b64, steps, warmup)
    b64.set_join_form(form)
    ms_joint = ms_form[form]
    t64, _, it64 = b64.state()
    t32, _, it32 = b32.state()
    out = {
        "metric": "batched 2D MHD mesh cell-updates/s, FP64 and FP32 instances joined in one graph",
        "value": cells * steps / (ms_joint / 1e3),
        "unit": "cell-updates/s",
        "ninst": [ninst, ninst],
        "mesh_cells": cells,
        "steps": steps,
        "warmup": warmup,
        "join_form": form,
        "ms_per_step_joined": ms_joint / steps,
        "ms_per_step_joint_kernels": ms_form[0] / steps,
        "ms_per_step_two_branches": ms_form[1] / steps,
        "join_stage_ms": {"joint_kernels": stage_joint, "two_branches": stage_forked},
        "ms_per_step_separate": ms_seq / steps,
        "value_separate": cells * steps / (ms_seq / 1e3),
        "fused_tile": [[32, 8], [16, 8]][b64.stage()[1]],
        "steps_done": [int(it64.min()), int(it32.min())],
        "config": {"workload": "uneven Orszag-Tang batch, each instance once in FP64 and once in FP32",
                   "sizes": f"{sizes[0]}..{sizes[-1]} step {sizes[1] - sizes[0]}", "beta": "U[0.5,10]",
                   "seed": seed},
    }
    b64.close()
    b32.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ninst", type=int, default=4096)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", choices=["fp64", "fp32", "both"], default="both")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--group-cells", type=int, default=0)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--stage", choices=["tuned", "three", "fused0", "fused1"], default="tuned",
                    help="the stage form: the tuner's choice, the three passes, or the fused kernel in tile shape 0/1")
    ap.add_argument("--joint", action="store_true", help="FP64 and FP32 batches of the same instances, joined")
    a = ap.parse_args(argv)
    if a.joint:
        r = run_joint(a.ninst, a.steps, a.warmup, seed=a.seed)
        print(json.dumps(r), flush=True)
        return [r]
    precs = {"fp64": [params.PREC_FP64], "fp32": [params.PREC_FP32],
             "both": [params.PREC_FP64, params.PREC_FP32]}[a.precision]
    res = []
    for p in precs:
        stage = {"tuned": None, "three": (False, 0), "fused0": (True, 0), "fused1": (True, 1)}[a.stage]
        r = run(a.ninst, a.steps, a.warmup, p, seed=a.seed, group_cells=a.group_cells, tune=not a.no_tune,
                stage=stage)
        print(json.dumps(r), flush=True)
        res.append(r)
    if len(res) == 2:
        print(json.dumps({"fp32_over_fp64": res[1]["value"] / res[0]["value"]}), flush=True)
    return res


if __name__ == "__main__":
    main()
