"""CPU oracle of the FNO surrogate (test infrastructure: only tests and the
benchmark's checks use it; the product never imports it).

A float64 numpy restatement of the network in sac_b200/csrc/fno/fno_net.cu,
written with FFTs (numpy.fft.rfft2 / irfft2 restricted to the kept modes)
instead of the DFT-matrix GEMMs of the CUDA path, so that it checks that
formulation independently.  It has no reference counterpart (the surrogate is a
library extension); its backward pass is pinned by finite differences in the
CPU tests.

Parameters come as the flat FP32 vector of sac_fno_get_params and the layout of
sac_fno_param_layout: P[width][cin], Pb, then per layer W[o][i], Wb, R.re and
R.im [kx][ky][i][o] (kx: the m1 lowest, then the m1 highest), then Q1[hidden][width],
Q1b, Q2[cout8][hidden] (rows >= cout zero), Q2b.
"""
from __future__ import annotations

import math

import numpy as np


# GELU in its tanh form (Hendrycks and Gimpel, "Gaussian Error Linear Units"):
# 0.5 x (1 + tanh(c0 (x + c1 x^3))), c0 = sqrt(2/pi), c1 = 0.044715
GELU_C0 = math.sqrt(2.0 / math.pi)
GELU_C1 = 0.044715


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(GELU_C0 * (x + GELU_C1 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_C0 * (x + GELU_C1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C0 * (1.0 + 3.0 * GELU_C1 * x * x)


class Layout:
    def __init__(self, width, layers, cin, cout, hidden, m1=24, m2=24):
        self.width, self.layers, self.cin, self.cout, self.hidden = width, layers, cin, cout, hidden
        self.m1, self.m2 = m1, m2
        self.cpad = (cout + 7) // 8 * 8
        off = 0
        segs = {}

        def seg(name, n):
            nonlocal off
            segs[name] = (off, n)
            off += (n + 7) // 8 * 8

        nm = 2 * m1 * m2
        seg("P", width * cin)
        seg("Pb", width)
        for l in range(layers):
            seg(f"W{l}", width * width)
            seg(f"Wb{l}", width)
            seg(f"Rr{l}", nm * width * width)
            seg(f"Ri{l}", nm * width * width)
        seg("Q1", hidden * width)
        seg("Q1b", hidden)
        seg("Q2", self.cpad * hidden)
        seg("Q2b", self.cpad)
        self.segs, self.n = segs, off

    def get(self, theta, name):
        o, n = self.segs[name]
        return theta[o:o + n]

    def unpack(self, theta):
        W, L, m1, m2 = self.width, self.layers, self.m1, self.m2
        t = np.asarray(theta, dtype=np.float64)
        p = {"P": self.get(t, "P").reshape(W, self.cin), "Pb": self.get(t, "Pb"),
             "Q1": self.get(t, "Q1").reshape(self.hidden, W), "Q1b": self.get(t, "Q1b"),
             "Q2": self.get(t, "Q2").reshape(self.cpad, self.hidden)[: self.cout],
             "Q2b": self.get(t, "Q2b")[: self.cout]}
        for l in range(L):
            p[f"W{l}"] = self.get(t, f"W{l}").reshape(W, W)
            p[f"Wb{l}"] = self.get(t, f"Wb{l}")
            rr = self.get(t, f"Rr{l}").reshape(2 * m1, m2, W, W)
            ri = self.get(t, f"Ri{l}").reshape(2 * m1, m2, W, W)
            p[f"R{l}"] = rr + 1j * ri
        return p

    def pack_grads(self, g):
        out = np.zeros(self.n)
        W, m1, m2 = self.width, self.m1, self.m2

        def put(name, arr):
            o, n = self.segs[name]
            out[o:o + n] = np.asarray(arr).reshape(-1)[:n]

        put("P", g["P"])
        put("Pb", g["Pb"])
        for l in range(self.layers):
            put(f"W{l}", g[f"W{l}"])
            put(f"Wb{l}", g[f"Wb{l}"])
            put(f"Rr{l}", g[f"R{l}"].real)
            put(f"Ri{l}", g[f"R{l}"].imag)
        put("Q1", g["Q1"])
        put("Q1b", g["Q1b"])
        q2 = np.zeros((self.cpad, self.hidden))
        q2[: self.cout] = g["Q2"]
        put("Q2", q2)
        q2b = np.zeros(self.cpad)
        q2b[: self.cout] = g["Q2b"]
        put("Q2b", q2b)
        return out


def _kx(S, m1):
    return np.concatenate([np.arange(m1), np.arange(S - m1, S)])


def spectral(v, R, m1, m2):
    """irfft2(R . rfft2(v)[kept modes]); v: [B][C][S][F]; R: [2m1][m2][i][o]."""
    B, C, S, F = v.shape
    kx = _kx(S, m1)
    Vh = np.fft.rfft2(v, axes=(2, 3))
    U = Vh[:, :, kx, :m2]                                  # [B][i][2m1][m2]
    O = np.einsum("bixy,xyio->boxy", U, R)
    full = np.zeros((B, R.shape[3], S, F // 2 + 1), dtype=complex)
    full[:, :, kx, :m2] = O
    return np.fft.irfft2(full, s=(S, F), axes=(2, 3)), U


def spectral_backward(dy, U, R, m1, m2):
    """Gradients of spectral() w.r.t. v and R given dy [B][o][S][F]."""
    B, O_, S, F = dy.shape
    kx = _kx(S, m1)
    w = np.where(np.arange(m2) == 0, 1.0, 2.0)
    G = np.fft.rfft2(dy, axes=(2, 3))[:, :, kx, :m2] * (w / (S * F))   # dL/dO (re + i im)
    dR = np.einsum("boxy,bixy->xyio", G, np.conj(U))
    GU = np.einsum("boxy,xyio->bixy", G, np.conj(R))
    full = np.zeros((B, R.shape[2], S, F), dtype=complex)
    full[:, :, kx, :m2] = GU
    dv = np.real(np.fft.ifft2(full, axes=(2, 3))) * (S * F)
    return dv, dR


def _pw(Wm, x, b=None):
    y = np.einsum("oi,bip->bop", Wm, x.reshape(x.shape[0], x.shape[1], -1))
    if b is not None:
        y = y + b[None, :, None]
    return y.reshape((x.shape[0], Wm.shape[0]) + x.shape[2:])


def forward(lay: Layout, theta, x):
    """x: [B][cin][S][F] float64 -> y [B][cout][S][F] and the tape for backward."""
    p = lay.unpack(theta)
    tape = {"x": x}
    v = _pw(p["P"], x, p["Pb"])
    tape["v0"] = v
    for l in range(lay.layers):
        sp, U = spectral(v, p[f"R{l}"], lay.m1, lay.m2)
        z = _pw(p[f"W{l}"], v, p[f"Wb{l}"]) + sp
        tape[f"U{l}"] = U
        tape[f"z{l}"] = z
        v = gelu(z) if l < lay.layers - 1 else z
        tape[f"v{l + 1}"] = v
    hp = _pw(p["Q1"], v, p["Q1b"])
    h = gelu(hp)
    tape["hp"], tape["h"] = hp, h
    y = _pw(p["Q2"], h, p["Q2b"])
    return y, tape


def backward(lay: Layout, theta, tape, dy):
    """Gradients (flat, in the parameter layout) of sum(dy * y)."""
    p = lay.unpack(theta)
    g = {}
    B = dy.shape[0]

    def wg(dout, inp):
        return np.einsum("bop,bip->oi", dout.reshape(B, dout.shape[1], -1), inp.reshape(B, inp.shape[1], -1))

    def bg(dout):
        return dout.sum(axis=(0, 2, 3))

    g["Q2"], g["Q2b"] = wg(dy, tape["h"]), bg(dy)
    dh = _pw(p["Q2"].T, dy)
    dhp = dh * gelu_grad(tape["hp"])
    g["Q1"], g["Q1b"] = wg(dhp, tape[f"v{lay.layers}"]), bg(dhp)
    dv = _pw(p["Q1"].T, dhp)
    for l in range(lay.layers - 1, -1, -1):
        dz = dv if l == lay.layers - 1 else dv * gelu_grad(tape[f"z{l}"])
        vin = tape[f"v{l}"]
        g[f"W{l}"], g[f"Wb{l}"] = wg(dz, vin), bg(dz)
        dsv, dR = spectral_backward(dz, tape[f"U{l}"], p[f"R{l}"], lay.m1, lay.m2)
        g[f"R{l}"] = dR
        dv = _pw(p[f"W{l}"].T, dz) + dsv
    g["P"], g["Pb"] = wg(dv, tape["x"]), bg(dv)
    return lay.pack_grads(g)


def bf16_round(a):
    """Round float values to the nearest bfloat16 (ties to even), as float64."""
    a32 = np.asarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)
