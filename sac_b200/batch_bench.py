"""Throughput of the batched path on uneven Orszag-Tang vortices.

    python -m sac_b200.batch_bench --ninst 4096 --steps 10 --warmup 3 --precision both

Builds the batch (sizes nx, ny drawn from {64, 96, ..., 512}, beta uniform in
[0.5, 10], seeded), lets the autotuner pick the update tile, replays the
captured RK4 step W times untimed, then times K steps with CUDA events on the
batch's stream.  Prints one JSON line per precision: mesh cell-updates/s over
the whole batch (every instance advances one step per replay, each with its own
dt), ms per step, the tile chosen, the device memory the batch holds and the
spread of the instances' simulated times.
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
    a = ap.parse_args(argv)
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
