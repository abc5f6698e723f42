"""The CPU oracle against physics the reference's equations must satisfy (CPU).

The reference ships no output vectors, so the oracle is pinned by invariants:
exact preservation of a zero perturbation over a stratified background, linear
wave speeds, the Brio-Wu wave structure and the boundary-fill rules."""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import params, problems

import _util


def test_zero_perturbation_is_exact():
    P = problems.stratified(n=(10, 8, 8), amp=0.0)
    o = _util.start(Oracle, P)
    _util.run(o, 10)
    w = o.download()
    assert np.all(w[..., : 2 * P.ndir + 2] == 0.0)


def _uniform_1d(nx, rho0=1.0, p0=1.0, B=(0.0, 0.0), gamma=5 / 3, nu=1.0):
    P = problems.brio_wu(nx=nx, nu=nu)
    v = problems.var_index(P.ndir)
    P.w[...] = 0.0
    P.w[..., v["rhob"]] = rho0
    P.w[..., v["bg0"] + 1] = B[0]
    P.w[..., v["bg0"] + 2] = B[1]
    P.w[..., v["eb"]] = p0 / (gamma - 1) + 0.5 * (B[0] ** 2 + B[1] ** 2)
    P.params.gamma = gamma
    P.params.user = params.USR_GRAVVISC
    return P, v


def _centroid(x, f):
    f = np.clip(f, 0, None)
    return float((x * f).sum() / f.sum())


def test_acoustic_pulse_speed():
    P, v = _uniform_1d(400)
    x = P.x[..., 0]
    pulse = 1e-4 * np.exp(-((x - 0.5) / 0.03) ** 2)
    P.w[..., v["rho"]] = pulse
    P.w[..., v["e"]] = pulse / (P.params.gamma - 1) * (5 / 3)  # adiabatic: p' = c^2 rho'
    o = _util.start(Oracle, P)
    t = 0.0
    it = 0
    while t < 0.15:
        dt = o.getdt(it)
        o.advect(dt, t, it)
        t += dt
        it += 1
    rho = o.download()[2:-2, v["rho"]]
    xm = x[2:-2]
    right = xm > 0.5
    cs = math.sqrt(5 / 3)
    assert abs(_centroid(xm[right], rho[right]) - (0.5 + cs * t)) < 0.01


def test_alfven_pulse_speed():
    P, v = _uniform_1d(400, B=(0.8, 0.0))
    x = P.x[..., 0]
    vy = 1e-4 * np.exp(-((x - 0.5) / 0.03) ** 2)
    P.w[..., v["m0"] + 2] = vy  # rho=1
    P.w[..., v["b0"] + 2] = -vy  # right-going Alfven wave: b_y = -sqrt(rho) v_y
    P.w[..., v["e"]] = 0.5 * vy ** 2 + 0.5 * vy ** 2
    o = _util.start(Oracle, P)
    t, it = 0.0, 0
    while t < 0.2:
        dt = o.getdt(it)
        o.advect(dt, t, it)
        t += dt
        it += 1
    my = o.download()[2:-2, v["m0"] + 2]
    xm = x[2:-2]
    assert abs(_centroid(xm, np.abs(my)) - (0.5 + 0.8 * t)) < 0.01


def test_briowu_structure():
    P = problems.brio_wu(nx=400)
    P.params.user = params.USR_GRAVVISC
    o = _util.start(Oracle, P)
    t, it = 0.0, 0
    while t < 0.1:
        dt = o.getdt(it)
        o.advect(dt, t, it)
        t += dt
        it += 1
    w = o.download()[2:-2]
    rho, x = w[:, 0], P.x[2:-2, 0]
    assert np.isfinite(w).all()
    # plateau between the compound wave and the contact, post-slow-shock state
    assert 0.64 < rho[(x > 0.48) & (x < 0.52)].mean() < 0.72
    assert 0.10 < rho[(x > 0.68) & (x < 0.74)].mean() < 0.14
    assert rho[x < 0.3].min() > 0.99 and abs(rho[x > 0.95].mean() - 0.125) < 2e-3


def test_courant_dt_uniform_state():
    P, v = _uniform_1d(100, B=(0.5, 0.3), nu=0.0)
    P.params.user = params.USR_NONE
    o = _util.start(Oracle, P)
    dt = o.getdt(0)
    g = 5 / 3
    cs2, B2 = g * 1.0, 0.5 ** 2 + 0.3 ** 2
    cf2 = B2 + cs2
    cmax = math.sqrt(0.5 * (cf2 + math.sqrt(cf2 ** 2 - 4 * cs2 * 0.25)))
    assert dt == pytest.approx(0.8 * (1 / 100) / cmax, rel=1e-12)


@pytest.mark.parametrize("kind", ["cont", "periodic", "symm", "asymm", "cont1", "contCD4"])
def test_boundary_rules(kind):
    P = problems.random_problem((8, 7), seed=2, types=[kind] * 4)
    o = _util.start(Oracle, P)
    w = o.download()
    a = w[..., 0]
    lo, hi = 2, 2 + 8 - 1
    if kind == "cont":
        assert np.all(a[:2, 2:-2] == a[2, 2:-2]) and np.all(a[-2:, 2:-2] == a[hi, 2:-2])
    elif kind == "periodic":
        np.testing.assert_array_equal(a[:2, 2:-2], a[hi - 1: hi + 1, 2:-2])
        np.testing.assert_array_equal(a[-2:, 2:-2], a[lo: lo + 2, 2:-2])
    elif kind in ("symm", "asymm"):
        s = -1.0 if kind == "asymm" else 1.0
        np.testing.assert_array_equal(a[1, 2:-2], s * a[2, 2:-2])
        np.testing.assert_array_equal(a[0, 2:-2], s * a[3, 2:-2])
    elif kind == "cont1":
        np.testing.assert_allclose(a[1, 2:-2], 2 * a[2, 2:-2] - a[3, 2:-2], rtol=1e-14)
    elif kind == "contCD4":
        np.testing.assert_array_equal(a[1, 2:-2], a[3, 2:-2])
        np.testing.assert_array_equal(a[0, 2:-2], a[4, 2:-2])


def test_fixed_boundary_holds_initial_ghosts():
    P = problems.random_problem((10, 8), seed=4, types=["fixed", "cont", "periodic", "periodic"])
    o = _util.start(Oracle, P)
    g0 = o.download()[:2].copy()
    _util.run(o, 5)
    np.testing.assert_array_equal(o.download()[:2, 2:-2, : 2 * P.ndir + 2], g0[:, 2:-2, : 2 * P.ndir + 2])
