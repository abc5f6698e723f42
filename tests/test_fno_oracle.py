"""The surrogate's CPU oracle (oracle/fno_ref.py) pinned on the CPU: its spectral
convolution against a brute-force DFT sum, and its backward pass against central
finite differences of its own forward pass."""
import numpy as np

from oracle import fno_ref


def _theta(lay, seed, scale=0.3):
    rng = np.random.default_rng(seed)
    t = rng.uniform(-scale, scale, lay.n)
    o, n = lay.segs["Q2"]
    q2 = t[o:o + n].reshape(lay.cpad, lay.hidden)
    q2[lay.cout:] = 0.0
    return t


def test_spectral_matches_brute_force_dft():
    rng = np.random.default_rng(0)
    B, C, S, F, m1, m2 = 1, 2, 50, 52, 24, 24
    v = rng.standard_normal((B, C, S, F))
    R = rng.standard_normal((2 * m1, m2, C, C)) + 1j * rng.standard_normal((2 * m1, m2, C, C))
    y, _ = fno_ref.spectral(v, R, m1, m2)
    s = np.arange(S)[:, None]
    f = np.arange(F)[None, :]
    kx = np.concatenate([np.arange(m1), np.arange(S - m1, S)])
    ref = np.zeros((B, C, S, F))
    for qi, k1 in enumerate(kx):
        for k2 in range(m2):
            e = np.exp(-2j * np.pi * (k1 * s / S + k2 * f / F))
            U = (v * e).sum(axis=(2, 3))                     # [B][i]
            O = U @ R[qi, k2]                                 # [B][o]
            w = 1.0 if k2 == 0 else 2.0
            ref += w * np.real(O[:, :, None, None] * np.conj(e)[None, None]) / (S * F)
    np.testing.assert_allclose(y, ref, rtol=1e-9, atol=1e-9)


def test_backward_matches_finite_differences():
    lay = fno_ref.Layout(width=16, layers=2, cin=16, cout=6, hidden=16)
    th = _theta(lay, 1)
    rng = np.random.default_rng(2)
    S = F = 56
    x = rng.standard_normal((2, 16, S, F))
    dy = rng.standard_normal((2, 6, S, F))
    y, tape = fno_ref.forward(lay, th, x)
    g = fno_ref.backward(lay, th, tape, dy)
    names = ["P", "Pb", "W0", "Wb0", "Rr0", "Ri0", "W1", "Rr1", "Ri1", "Q1", "Q1b", "Q2", "Q2b"]
    h = 1e-6
    for name in names:
        o, n = lay.segs[name]
        if name.startswith("Q2"):
            n = lay.cout * (lay.hidden if name == "Q2" else 1)
        for k in rng.choice(n, 3, replace=False):
            i = o + int(k)
            tp, tm = th.copy(), th.copy()
            tp[i] += h
            tm[i] -= h
            lp = (fno_ref.forward(lay, tp, x)[0] * dy).sum()
            lm = (fno_ref.forward(lay, tm, x)[0] * dy).sum()
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (name, k, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.00390625, 1.01171875, -3.14159, 65504.0])
    r = fno_ref.bf16_round(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625
    assert abs(r[3] + 3.140625) < 1e-12
