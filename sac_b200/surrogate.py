"""FNO surrogate of the 2D flux-tube workload: data, training, judged roll-out.

    python -m sac_b200.surrogate --ntrain 2000 --ntest 200 --epochs 4 --out fno_run

* Data: FP32 solver trajectories of the flux tube (sac_b200.problems.flux_tube,
  256 x 256) with seeded drivers, A log-uniform in [1e-4, 1e-2] and omega uniform
  in [0.5, 2] x the acoustic cut-off, advanced together by the batched solver
  with a fixed dt; the state is gathered on the device every `window` steps.
  Sample k of trajectory n is (w_k / A, (w_{k+1} - w_k) / A), both BF16.
* Network: libsacfno.so (4 Fourier layers, width 32, 24 x 24 modes, BF16 with
  FP32 accumulation), trained with its own forward/backward kernels and Adam on
  the per-channel normalised increments.  Inputs: the six normalised perturbed
  fields, sin(omega t), cos(omega t), omega/omega_ac - 1.25, log10(A) + 3 and the
  two coordinates.
* Judge: the roll-out advances every held-out driver by the surrogate, one call
  per window; every M-th call the plain solver re-runs that window from the same
  start state, and the surrogate's window is rejected (replaced by the solver's)
  when its relative L2 exceeds `tol` or its div B / energy drift exceed the
  stated bounds.  The result is compared with the plain solver's own final state.

PyTorch serves here only as the training driver's container of device buffers
and for the judge's reductions; every network pass is a libsacfno.so kernel and
every solver step a libsacgpu.so kernel.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import batch as sbatch
from . import fno_abi, params, problems

NST = 6        # rho, m1, m2, e, b1, b2 (2D, ndir 2)
NFEAT = 4      # sin(wt), cos(wt), omega/omega_ac - 1.25, log10(A) + 3


def _torch():
    import torch
    return torch


# ---------------------------------------------------------------------------
# drivers and the batched solver
# ---------------------------------------------------------------------------
def drivers(n, seed, omega_ac):
    rng = np.random.default_rng(seed)
    A = 10.0 ** rng.uniform(-4.0, -2.0, n)
    om = rng.uniform(0.5, 2.0, n) * omega_ac
    return A, om


def make_solver(A, om, n=(256, 256), dtpar=None, precision=params.PREC_FP32, group_cells=0):
    P0 = problems.flux_tube(n)
    prm = P0.params
    prm.precision = precision
    if dtpar is not None:
        prm.dtpar = dtpar
    ninst = len(A)
    b = sbatch.Batch(prm, 2, 2, [n] * ninst, group_cells=group_cells)
    b.set_grid(np.concatenate([P0.x.reshape(-1, order="F")] * ninst))
    b.set_boundaries(P0.typeB)
    w0 = P0.w.reshape(-1, order="F")
    chunk = 64
    for i0 in range(0, ninst, chunk):
        k = min(chunk, ninst - i0)
        b.upload(np.concatenate([w0] * k), i0, k)
    b.set_driver(A, om)
    b.getboundary()
    b.tune()  # the stage form and tile the batch runs fastest with (the fused 2D stage)
    return b, P0


def stable_dt(n=(256, 256), nsteps=48, safety=0.6, seed=123):
    """A fixed dt below the adaptive (Courant and viscous) limits the solver takes
    on a few strongly driven instances over the first steps."""
    omega_ac = problems.flux_tube(n).meta["omega_ac"]
    A = np.full(4, 1e-2)
    om = np.array([0.5, 1.0, 1.5, 2.0]) * omega_ac
    b, _ = make_solver(A, om, n=n)
    dmin = 1e99
    for _ in range(nsteps):
        b.advance(1)
        dmin = min(dmin, float(b.state()[1].min()))
    b.close()
    return safety * dmin


# ---------------------------------------------------------------------------
# data
# ---------------------------------------------------------------------------
class Dataset:
    """X[n][k] = w_k / A_n and D[n][k] = (w_{k+1} - w_k) / A_n on the device (BF16)."""

    def __init__(self, ntraj, nwin, S=256, F=256, device="cuda"):
        torch = _torch()
        self.X = torch.empty(ntraj, nwin, NST, S, F, dtype=torch.bfloat16, device=device)
        self.D = torch.empty(ntraj, nwin, NST, S, F, dtype=torch.bfloat16, device=device)
        self.A = np.zeros(ntraj)
        self.om = np.zeros(ntraj)
        self.t0 = np.zeros(nwin)
        self.ntraj, self.nwin = ntraj, nwin


def generate(ds: Dataset, A, om, dt, window, n=(256, 256), chunk=500, log=print):
    """Fill ds with solver trajectories (FP32 batched solver, fixed dt)."""
    torch = _torch()
    S, F = n[1], n[0]
    t0 = time.time()
    for c0 in range(0, ds.ntraj, chunk):
        k = min(chunk, ds.ntraj - c0)
        b, _ = make_solver(A[c0:c0 + k], om[c0:c0 + k], n=n, dtpar=dt)
        cur = torch.empty(k, NST, S, F, dtype=torch.float32, device="cuda")
        nxt = torch.empty_like(cur)
        inv = torch.tensor(1.0 / A[c0:c0 + k], dtype=torch.float32, device="cuda").view(k, 1, 1, 1)
        stream = torch.cuda.ExternalStream(b.stream())
        b.gather(cur.data_ptr(), "f32")
        for w in range(ds.nwin):
            b.advance(window)
            b.gather(nxt.data_ptr(), "f32")
            with torch.cuda.stream(stream):
                ds.X[c0:c0 + k, w] = (cur * inv).to(torch.bfloat16)
                ds.D[c0:c0 + k, w] = ((nxt - cur) * inv).to(torch.bfloat16)
                cur, nxt = nxt, cur
        b.synchronize()
        t, _, it = b.state()
        if not np.isfinite(cur.cpu().numpy()).all():
            raise RuntimeError("non-finite solver state in the training data")
        ds.A[c0:c0 + k], ds.om[c0:c0 + k] = A[c0:c0 + k], om[c0:c0 + k]
        b.close()
        log(f"generated {c0 + k}/{ds.ntraj} trajectories, t_end={t[0]:.4f}, {time.time() - t0:.1f} s")
    ds.t0 = np.arange(ds.nwin) * window * dt


def channel_scales(ds: Dataset, nsample=64):
    torch = _torch()
    idx = torch.randperm(ds.ntraj)[:nsample]
    x = ds.X[idx].float()
    d = ds.D[idx].float()
    sx = x.pow(2).mean(dim=(0, 1, 3, 4)).sqrt().clamp_min(1e-12)
    sd = d.pow(2).mean(dim=(0, 1, 3, 4)).sqrt().clamp_min(1e-12)
    return sx.cpu().numpy(), sd.cpu().numpy()


def features_host(A, om, t, omega_ac):
    f = np.stack([np.sin(om * t), np.cos(om * t), om / omega_ac - 1.25, np.log10(A) + 3.0], axis=-1)
    return f.astype(np.float32)


# ---------------------------------------------------------------------------
# training
# ---------------------------------------------------------------------------
class Surrogate:
    def __init__(self, S=256, F=256, batch=16, seed=0, width=32, layers=4, hidden=128, infer_batch=None):
        """batch: the training minibatch; infer_batch: the samples per inference
        call of predict (default: batch)."""
        torch = _torch()
        self.BI = infer_batch or batch
        nmax = max(batch, self.BI)
        self.net = fno_abi.Net(S=S, F=F, width=width, layers=layers, hidden=hidden, cin=16, cout=NST,
                               max_batch=nmax, seed=seed)
        self.B, self.S, self.F = batch, S, F
        self.stream = torch.cuda.ExternalStream(self.net.stream)
        dev = "cuda"
        self.x = torch.zeros(nmax, 16, S, F, dtype=torch.bfloat16, device=dev)
        self.y = torch.zeros(nmax, NST, S, F, dtype=torch.float32, device=dev)
        self.dy = torch.zeros(batch, self.net.cpad, S, F, dtype=torch.bfloat16, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.tgt = torch.zeros(batch, NST, S, F, dtype=torch.bfloat16, device=dev)
        self.scale = torch.zeros(batch * NST, dtype=torch.float32, device=dev)
        self.feat = torch.zeros(batch * NFEAT, dtype=torch.float32, device=dev)
        self.sx = np.ones(NST)
        self.sd = np.ones(NST)
        self.step = 0
        self.omega_ac = problems.flux_tube((F, S)).meta["omega_ac"]

    def set_scales(self, sx, sd):
        self.sx, self.sd = np.asarray(sx, dtype=np.float64), np.asarray(sd, dtype=np.float64)

    def _load_batch(self, ds, idx):
        torch = _torch()
        n = idx[:, 0]
        k = idx[:, 1]
        B = len(idx)
        with torch.cuda.stream(self.stream):
            ni = torch.as_tensor(n, device="cuda")
            ki = torch.as_tensor(k, device="cuda")
            st = ds.X[ni, ki]
            self.tgt[:B] = (ds.D[ni, ki].float() / torch.as_tensor(self.sd, dtype=torch.float32,
                                                                   device="cuda").view(1, NST, 1, 1)
                            ).to(torch.bfloat16)
            self.scale[:B * NST] = torch.as_tensor(np.tile(1.0 / self.sx, B), dtype=torch.float32, device="cuda")
            f = features_host(ds.A[n], ds.om[n], ds.t0[k], self.omega_ac)
            self.feat[:B * NFEAT] = torch.as_tensor(f.reshape(-1), device="cuda")
            self._st = st.contiguous()
        self.net.features(self._st.data_ptr(), True, self.scale.data_ptr(), self.feat.data_ptr(), NFEAT,
                          self.x.data_ptr(), B, NST)

    def train(self, ds, epochs=2, lr=1e-3, wd=1e-4, clip=1.0, val_frac=0.05, log=print, seed=0,
              max_steps=None, time_limit=None):
        torch = _torch()
        rng = np.random.default_rng(seed)
        pairs = np.array([(n, k) for n in range(ds.ntraj) for k in range(ds.nwin)])
        rng.shuffle(pairs)
        nval = max(self.B, int(len(pairs) * val_frac))
        val, tr = pairs[:nval], pairs[nval:]
        steps_per_epoch = len(tr) // self.B
        total = int(steps_per_epoch * epochs)
        if max_steps is not None:
            total = min(total, int(max_steps))
        hist = []
        t0 = time.time()
        for it in range(total):
            if it % steps_per_epoch == 0:
                rng.shuffle(tr)
            j = it % steps_per_epoch
            idx = tr[j * self.B:(j + 1) * self.B]
            self._load_batch(ds, idx)
            self.step += 1
            lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * it / total))
            with torch.cuda.stream(self.stream):
                self.loss.zero_()
            self.net.zero_grad()
            self.net.forward(self.x.data_ptr(), self.y.data_ptr(), self.B)
            self.net.mse(self.y.data_ptr(), self.tgt.data_ptr(), self.dy.data_ptr(), self.loss.data_ptr(), self.B)
            self.net.backward(self.dy.data_ptr())
            self.net.adam(lr_t, self.step, wd=wd, clip=clip)
            if it % 200 == 0 or it == total - 1:
                self.net.check()
                l = float(self.loss.item())
                hist.append((it, l))
                log(f"step {it}/{total} loss {l:.4e} lr {lr_t:.2e} {time.time() - t0:.1f} s")
            if time_limit and time.time() - t0 > time_limit:
                log(f"time limit reached at step {it}")
                break
        self.net.check()
        return hist, self.evaluate_loss(ds, val)

    def evaluate_loss(self, ds, pairs):
        """Mean loss and the relative L2 of the predicted increments on pairs."""
        torch = _torch()
        tot, rel, nb = 0.0, [], 0
        for j in range(0, len(pairs) - self.B + 1, self.B):
            idx = pairs[j:j + self.B]
            self._load_batch(ds, idx)
            with torch.cuda.stream(self.stream):
                self.loss.zero_()
            self.net.forward(self.x.data_ptr(), self.y.data_ptr(), self.B)
            self.net.mse(self.y.data_ptr(), self.tgt.data_ptr(), self.dy.data_ptr(), self.loss.data_ptr(), self.B)
            torch.cuda.synchronize()
            tot += float(self.loss.item())
            t = self.tgt.float()
            e = (self.y - t).pow(2).sum(dim=(1, 2, 3)).sqrt() / t.pow(2).sum(dim=(1, 2, 3)).sqrt().clamp_min(1e-30)
            rel += e.cpu().tolist()
            nb += 1
        return {"val_loss": tot / max(nb, 1), "val_rel_l2_increment": float(np.mean(rel)) if rel else None}

    # -----------------------------------------------------------------------
    def predict(self, state, A, om, t):
        """Advance the states by one window in place.  state: torch float32
        [n][6][S][F] (raw perturbation, packed layout of sac_batch_gather)."""
        torch = _torch()
        n = state.shape[0]
        # the window's scales and features of all n instances in one copy each, so
        # that the host enqueues the chunks without waiting on the stream
        sc = np.concatenate([np.tile(1.0 / self.sx, n) / np.repeat(A, NST), np.tile(self.sd, n) * np.repeat(A, NST)])
        f = features_host(A, om, np.full(n, t), self.omega_ac).reshape(-1)
        with torch.cuda.stream(self.stream):
            scd = torch.as_tensor(sc, dtype=torch.float32).pin_memory().to("cuda", non_blocking=True)
            fd = torch.as_tensor(f, dtype=torch.float32).pin_memory().to("cuda", non_blocking=True)
        fsz = 4  # bytes per float32
        for i0 in range(0, n, self.BI):
            B = min(self.BI, n - i0)
            blk = state[i0:i0 + B]
            self.net.features(blk.data_ptr(), False, scd.data_ptr() + i0 * NST * fsz, fd.data_ptr() + i0 * NFEAT * fsz,
                              NFEAT, self.x.data_ptr(), B, NST)
            self.net.infer(self.x.data_ptr(), self.y.data_ptr(), B)
            self.net.apply(blk.data_ptr(), self.y.data_ptr(), scd.data_ptr() + (n + i0) * NST * fsz, B, NST)
        self._keep = (scd, fd)  # alive until the stream has used them

    def save(self, path):
        np.savez(path, params=self.net.get_params(), sx=self.sx, sd=self.sd)

    def load(self, path):
        d = np.load(path)
        self.net.set_params(d["params"])
        self.set_scales(d["sx"], d["sd"])


# ---------------------------------------------------------------------------
# judged roll-out
# ---------------------------------------------------------------------------
def divb(state, dx1, dx2):
    """Fourth-order div b' on the interior (x1 fastest): [n] RMS values."""
    b1 = state[:, 4]
    b2 = state[:, 5]
    d1 = (-b1[:, :, 4:] + 8 * b1[:, :, 3:-1] - 8 * b1[:, :, 1:-3] + b1[:, :, :-4]) / (12 * dx1)
    d2 = (-b2[:, 4:, :] + 8 * b2[:, 3:-1, :] - 8 * b2[:, 1:-3, :] + b2[:, :-4, :]) / (12 * dx2)
    dv = d1[:, 2:-2, :] + d2[:, :, 2:-2]
    return dv.pow(2).mean(dim=(1, 2)).sqrt()


def energy(state):
    return state[:, 3].sum(dim=(1, 2))


def energy_drift(state, check):
    """|sum e'_surrogate - sum e'_solver| / sum |e'_solver|  per instance"""
    return (energy(state) - energy(check)).abs() / check[:, 3].abs().sum(dim=(1, 2)).clamp_min(1e-30)


def rel_l2(a, b):
    n = a.shape[0]
    return ((a - b).reshape(n, -1).norm(dim=1) / b.reshape(n, -1).norm(dim=1).clamp_min(1e-30))


def rollout(sur: Surrogate, A, om, dt, window, nwin, M=16, tol=1e-3, divb_tol=1e-3, energy_tol=1e-3,
            n=(256, 256), solver_windows=0, log=print):
    """Judged surrogate roll-out and the plain solver's own run on the same
    drivers; returns errors and device times (CUDA events).  The first
    `solver_windows` windows (growth from rest, where the surrogate's relative
    error is largest) are taken by the plain solver, inside the timed region."""
    torch = _torch()
    S, F = n[1], n[0]
    ninst = len(A)
    # the plain solver alone, timed
    ref, _ = make_solver(A, om, n=n, dtpar=dt)
    rs = torch.cuda.ExternalStream(ref.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ref.advance(1)  # graph capture and warm-up outside the timing
    ref.synchronize()
    ref.close()
    ref, P0 = make_solver(A, om, n=n, dtpar=dt)
    rs = torch.cuda.ExternalStream(ref.stream())
    ref.advance(0)
    torch.cuda.synchronize()
    e0.record(rs)
    ref.advance(window * nwin)
    e1.record(rs)
    e1.synchronize()
    solver_ms = e0.elapsed_time(e1)
    truth = torch.empty(ninst, NST, S, F, dtype=torch.float32, device="cuda")
    ref.gather(truth.data_ptr(), "f32")
    ref.synchronize()
    ref.close()
    dx1 = problems.flux_tube(n).x[1, 0, 0] - problems.flux_tube(n).x[0, 0, 0]
    dx2 = problems.flux_tube(n).x[0, 1, 1] - problems.flux_tube(n).x[0, 0, 1]
    # the surrogate with the judge: the plain solver re-runs a window with the same
    # fixed dt as the reference run (the driver enters each RK4 step at the step's
    # start time, a first-order treatment, so runs with different dt differ by
    # percents early on); tmax lands it on the window's end and keeps instances
    # that are already there untouched
    judge, _ = make_solver(A, om, n=n, dtpar=dt)
    judge.advance(0)
    state = torch.zeros(ninst, NST, S, F, dtype=torch.float32, device="cuda")
    judge.gather(state.data_ptr(), "f32")
    judge.synchronize()
    start = torch.empty_like(state)
    check = torch.empty_like(state)
    ckpt = state.clone()
    t_ck = 0.0
    judge_steps = 0
    rejected, judged, worst = 0, 0, 0.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record()
    if solver_windows > 0:
        judge.advance(window * solver_windows)
        judge.gather(state.data_ptr(), "f32")
        judge.synchronize()
        ckpt.copy_(state)
        t_ck = solver_windows * window * dt
    for k in range(solver_windows, nwin):
        t, t_next = k * window * dt, (k + 1) * window * dt
        judged_now = (k + 1) % M == 0
        if judged_now:
            start.copy_(state)
        torch.cuda.synchronize()
        sur.predict(state, A, om, t)
        torch.cuda.synchronize()
        if not judged_now:
            continue
        # the plain solver re-runs this window from the same start state
        judge.scatter(start.data_ptr(), "f32")
        judge.getboundary()
        judge.set_time(np.full(ninst, t), np.full(ninst, 1, dtype=np.int32))
        judge_steps += judge.advance_to(np.full(ninst, t_next))
        judge.gather(check.data_ptr(), "f32")
        judge.synchronize()
        err = rel_l2(state, check)
        ddiv = (divb(state, dx1, dx2) - divb(check, dx1, dx2)).abs() / \
            state[:, 4:6].reshape(ninst, -1).norm(dim=1).clamp_min(1e-30) * math.sqrt(S * F) * dx1
        den = energy_drift(state, check)
        bad = (err > tol) | (ddiv > divb_tol) | (den > energy_tol)
        nbad = int(bad.sum().item())
        judged += ninst
        rejected += nbad
        worst = max(worst, float(err.max().item()))
        if nbad:
            # rejected: roll those instances back to the last accepted state and let
            # the plain solver advance them over the M windows since then (the
            # accepted ones start at t_next and stay untouched)
            judge.scatter(ckpt.data_ptr(), "f32")
            judge.getboundary()
            bn = bad.cpu().numpy()
            judge.set_time(np.where(bn, t_ck, t_next), np.full(ninst, 1, dtype=np.int32))
            judge_steps += judge.advance_to(np.full(ninst, t_next))
            judge.gather(check.data_ptr(), "f32")
            judge.synchronize()
            state[bad] = check[bad]
        ckpt.copy_(state)
        t_ck = t_next
    s1.record()
    s1.synchronize()
    sur_ms = s0.elapsed_time(s1)
    wall = time.perf_counter() - t0
    judge.close()
    final = rel_l2(state, truth).cpu().numpy()
    out = {"ninst": ninst, "windows": nwin, "window_steps": window, "M": M, "tol": tol,
           "solver_ms": solver_ms, "surrogate_ms": sur_ms, "surrogate_wall_s": wall,
           "speedup": solver_ms / sur_ms, "final_rel_l2_mean": float(final.mean()),
           "final_rel_l2_max": float(final.max()), "final_rel_l2_median": float(np.median(final)),
           "judged": judged, "rejected": rejected, "worst_judged_rel_l2": worst,
           "judge_solver_steps": judge_steps, "solver_windows": solver_windows}
    log(json.dumps(out))
    return out


def persistence_error(ds: Dataset, pairs):
    """Relative L2 of the 'no change' prediction over one window (what the
    surrogate has to beat): |D| / |X| on the pairs."""
    vals = []
    for n, k in pairs:
        x = ds.X[n, k].float()
        d = ds.D[n, k].float()
        vals.append(float(d.norm() / (x + d).norm().clamp_min(1e-30)))
    return float(np.mean(vals))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ntrain", type=int, default=2000)
    ap.add_argument("--ntest", type=int, default=200)
    ap.add_argument("--steps", type=int, default=512)
    ap.add_argument("--window", type=int, default=16)
    ap.add_argument("--epochs", type=float, default=2)
    ap.add_argument("--max-steps", type=int, default=None)
    ap.add_argument("--time-limit", type=float, default=None)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--infer-batch", type=int, default=64, help="samples per inference call in the roll-outs")
    ap.add_argument("--M", type=int, default=16)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--weights", default=None, help="skip data and training; load these weights")
    ap.add_argument("--dt", type=float, default=None, help="the fixed dt of the trajectories")
    ap.add_argument("--solver-windows", type=int, default=2,
                    help="windows from rest taken by the plain solver in the second set of roll-outs")
    a = ap.parse_args(argv)
    torch = _torch()
    torch.cuda.init()
    from . import build
    build.build()
    build.build_fno()
    n = (a.n, a.n)
    log = lambda m: print(m, flush=True)  # noqa: E731
    omega_ac = problems.flux_tube(n).meta["omega_ac"]
    dt = a.dt if a.dt else stable_dt(n)
    nwin = a.steps // a.window
    log(f"fixed dt {dt:.4e}, {nwin} windows of {a.window} steps")
    sur = Surrogate(S=n[1], F=n[0], batch=a.batch, seed=a.seed, infer_batch=a.infer_batch)
    hist, val, gen_s = [], {}, 0.0
    if a.weights:
        sur.load(a.weights)
    else:
        ds = Dataset(a.ntrain, nwin, S=n[1], F=n[0])
        A, om = drivers(a.ntrain, a.seed, omega_ac)
        t0 = time.time()
        generate(ds, A, om, dt, a.window, n=n, log=log)
        gen_s = time.time() - t0
        sx, sd = channel_scales(ds)
        sur.set_scales(sx, sd)
        hist, val = sur.train(ds, epochs=a.epochs, lr=a.lr, log=log, max_steps=a.max_steps,
                              time_limit=a.time_limit)
        rng = np.random.default_rng(1)
        sample = [(int(rng.integers(ds.ntraj)), int(rng.integers(ds.nwin))) for _ in range(64)]
        val["persistence_rel_l2_state"] = persistence_error(ds, sample)
        log(json.dumps(val))
        del ds
        torch.cuda.empty_cache()
    At, omt = drivers(a.ntest, a.seed + 1000, omega_ac)
    runs = []
    for M, tol, sw in ((a.M, 1e-3, 0), (a.M, 2e-2, 0), (10 ** 9, 1e-3, 0), (a.M, 1e-3, a.solver_windows),
                       (a.M, 2e-2, a.solver_windows), (10 ** 9, 1e-3, a.solver_windows)):
        r = rollout(sur, At, omt, dt, a.window, nwin, M=M, tol=tol, n=n, solver_windows=sw, log=log)
        runs.append(r)
    res = {"rollouts": runs, "train": val, "generate_s": gen_s, "dt": dt, "ntrain": a.ntrain,
           "train_steps": sur.step}
    if a.out:
        os.makedirs(os.path.dirname(a.out) or ".", exist_ok=True)
        sur.save(a.out + "_weights.npz")
        with open(a.out + ".json", "w") as f:
            json.dump({"result": res, "loss_history": hist}, f, indent=1)
    return res


if __name__ == "__main__":
    main()
