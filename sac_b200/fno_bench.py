"""Throughput of the FNO kernels (libsacfno.so) on the surrogate's 256 x 256 grid.

    python -m sac_b200.fno_bench [--batch 16] [--iters 20] [--train]

Times the forward pass (and with --train a full training step: forward, loss,
backward, Adam) with CUDA events on the network's stream after warm-up, and
reports samples/s, the FLOPs of the network per sample, the achieved TFLOP/s and
the algorithmic bytes of the forward pass per sample.
"""
from __future__ import annotations

import argparse
import json

from . import fno_abi


def flops_per_sample(S=256, F=256, W=32, L=4, H=128, cin=16, cout=6, J=48, R=96):
    """Multiply-adds x 2 of the GEMMs and the mode mixing, forward pass."""
    P = S * F
    f = 2 * P * cin * W                                  # lift
    per_layer = (2 * W * S * F * J                       # F1
                 + 2 * W * J * S * R                     # F2
                 + 8 * (2 * 24 * 24) * W * W             # mixing (complex)
                 + 2 * W * J * R * S                     # F4
                 + 2 * W * S * J * F                     # F5
                 + 2 * P * W * W)                        # F6
    f += L * per_layer
    f += 2 * P * W * H + 2 * P * H * cout                # projection
    return f


def bytes_per_sample(S=256, F=256, W=32, L=4, H=128, cin=16, cout=6):
    """Compulsory DRAM bytes of one forward pass: the input, every layer's BF16
    activation written once and read once, the projection's hidden activation
    written and read once, the FP32 output (weights and DFT tables are shared by
    the batch and omitted)."""
    P = S * F
    return P * (cin * 2 + L * W * 2 * 2 + W * 2 + H * 2 * 2 + cout * 4)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--train", action="store_true")
    a = ap.parse_args(argv)
    import torch

    from . import build
    build.build_fno()
    B = a.batch
    net = fno_abi.Net(max_batch=B, seed=0)
    st = torch.cuda.ExternalStream(net.stream)
    x = torch.randn(B, 16, 256, 256, device="cuda").to(torch.bfloat16)
    y = torch.zeros(B, 6, 256, 256, device="cuda")
    tgt = torch.randn(B, 6, 256, 256, device="cuda").to(torch.bfloat16)
    dy = torch.zeros(B, net.cpad, 256, 256, dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()

    def fwd():
        net.infer(x.data_ptr(), y.data_ptr(), B)

    step = [0]

    def train():
        step[0] += 1
        net.zero_grad()
        net.forward(x.data_ptr(), y.data_ptr(), B)
        net.mse(y.data_ptr(), tgt.data_ptr(), dy.data_ptr(), loss.data_ptr(), B)
        net.backward(dy.data_ptr())
        net.adam(1e-4, step[0])

    fn = train if a.train else fwd
    for _ in range(a.warmup):
        fn()
    net.check()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(a.iters):
        fn()
    e1.record(st)
    e1.synchronize()
    net.check()
    ms = e0.elapsed_time(e1) / a.iters
    fl = flops_per_sample() * (3 if a.train else 1)
    out = {"mode": "train step" if a.train else "inference forward", "batch": B, "ms_per_call": ms,
           "samples_per_s": B / (ms / 1e3), "flops_per_sample": fl, "tflops": fl * B / (ms / 1e3) / 1e12,
           "forward_bytes_per_sample": bytes_per_sample(),
           "forward_gbs": (bytes_per_sample() * B / (ms / 1e3) / 1e9) if not a.train else None}
    print(json.dumps(out), flush=True)
    net.close()
    return out


if __name__ == "__main__":
    main()
