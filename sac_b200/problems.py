"""Synthetic workloads: initial states, grids, boundaries and parameters.

Layouts follow the reference: state w(ixG^T,nw) in Fortran order with variables
rho m1..m_ndir e b1..b_ndir eb rhob bg1..bg_ndir (src/vacpar.t.mhd:9-13), two
ghost layers (src/vacdef.t:23), x1 as the vertical axis where gravity acts (the
convention of src/vacusr.f:1294-1331).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .params import (USR_NONE, USR_STRAT, USR_TUBE, SacParams, make_params,
                     pack_typeB)

DIXB = 2


def var_index(ndir):
    e = ndir + 1
    return dict(rho=0, m0=0, e=e, b0=e, eb=e + ndir + 1, rhob=e + ndir + 2, bg0=e + ndir + 2,
                nw=3 * ndir + 4)


@dataclass
class Problem:
    name: str
    ndim: int
    ndir: int
    nx: tuple
    params: SacParams
    x: np.ndarray
    w: np.ndarray
    typeB: list
    tmax: float = 1e99
    nsteps: int = 0
    meta: dict = field(default_factory=dict)
    # user boundary regions (ixBmin, ixBmax, idimB, upperB) for Context.set_boundaries,
    # one per entry of typeB; None: the 2*ndim default regions
    regions: tuple = None

    @property
    def nw(self):
        return 3 * self.ndir + 4

    @property
    def ixGhi(self):
        return tuple(n + 2 * DIXB for n in self.nx)

    @property
    def ixM(self):
        lo = [DIXB + 1] * 3
        hi = [n + DIXB for n in self.nx] + [1] * (3 - self.ndim)
        lo = lo[: self.ndim] + [1] * (3 - self.ndim)
        return tuple(lo + hi)

    @property
    def typeB_packed(self):
        return pack_typeB(self.typeB)

    @property
    def nB(self):
        return len(self.typeB) if self.regions is not None else 2 * self.ndim

    @property
    def ncells(self):
        return int(np.prod(self.nx))


def cell_centres(nx, lo, hi):
    """Cell-centred coordinates on the full grid (ghosts included, extended linearly)."""
    d = (hi - lo) / nx
    i = np.arange(-DIXB, nx + DIXB)
    return lo + (i + 0.5) * d


def make_grid(nx, lows, highs):
    axes = [cell_centres(n, a, b) for n, a, b in zip(nx, lows, highs)]
    mesh = np.meshgrid(*axes, indexing="ij")
    x = np.stack(mesh, axis=-1)
    return np.asfortranarray(x)


def empty_state(nx, ndir):
    shape = tuple(n + 2 * DIXB for n in nx)
    return np.zeros(shape + (3 * ndir + 4,), order="F")


def uniform_types(ndim, nw, t):
    return [[t] * nw for _ in range(2 * ndim)]


# ---------------------------------------------------------------------------
# Brio-Wu shock tube (the reference's inipar/briowu-test12.py set-up)
# ---------------------------------------------------------------------------
def brio_wu(nx=800, courantpar=0.8, tmax=0.1, typeadvance="fourstep", nu=1.0) -> Problem:
    """1D ideal-MHD Riemann problem: gamma=2, b1=0.75, left (rho,p,b2)=(1,1,1),
    right (0.125,0.1,-1), split at the middle cell, zero background, cont bounds.
    Values match inipar/briowu-test12.py:19-73 (Ep = p/(gamma-1) + b^2/2)."""
    ndim, ndir = 1, 2
    gamma = 2.0
    x = make_grid((nx,), (0.0,), (1.0,))
    w = empty_state((nx,), ndir)
    v = var_index(ndir)
    half = nx // 2
    m = slice(DIXB, DIXB + nx)
    rho = np.where(np.arange(nx) < half, 1.0, 0.125)
    p = np.where(np.arange(nx) < half, 1.0, 0.1)
    b1, b2 = 0.75, np.where(np.arange(nx) < half, 1.0, -1.0)
    w[m, v["rho"]] = rho
    w[m, v["e"]] = p / (gamma - 1.0) + 0.5 * (b1 * b1 + b2 * b2)
    w[m, v["b0"] + 1] = b1
    w[m, v["b0"] + 2] = b2
    # hyperdiffusion with the viscous dt limit (gravity module, zero gravity):
    # at Courant 0.8 the Courant limit alone lets the shock blow up
    from .params import USR_GRAVVISC
    prm = make_params(gamma=gamma, nu=nu, courantpar=courantpar, typeadvance=typeadvance,
                      user=USR_GRAVVISC, grav=(0.0, 0.0, 0.0))
    return Problem("briowu", ndim, ndir, (nx,), prm, x, w, uniform_types(ndim, v["nw"], "cont"), tmax=tmax)


# ---------------------------------------------------------------------------
# gravitationally stratified atmosphere (x1 vertical)
# ---------------------------------------------------------------------------
def stratified(n=(128, 128, 128), height=1.5, H=0.3, B0=0.3, gamma=5.0 / 3.0, amp=None,
               omega=2 * math.pi / 0.3, z0=0.1, dz0=0.05, sigma=0.05, nu=1.0,
               typeadvance="fourstep", courantpar=0.8, perturb=None, seed=0, nsteps=500) -> Problem:
    """Isothermal hydrostatic background rho_b=exp(-z/H), p_b=rho_b*g*H (g=1),
    uniform vertical field B_b=B0 along x1, gamma=5/3; zero initial perturbation
    (optionally a seeded random-mode perturbation); fixed lower / open upper
    boundary in x1, periodic x2 and x3; a vertical velocity driver
    v = A sin(omega t) exp(-r^2/sigma^2) exp(-(z-z0)^2/dz0^2), A = 1e-3 c_s."""
    ndim = len(n)
    ndir = 3 if ndim == 3 else 2
    lows = (0.0,) + (0.0,) * (ndim - 1)
    highs = (height,) + (1.0,) * (ndim - 1)
    x = make_grid(n, lows, highs)
    w = empty_state(n, ndir)
    v = var_index(ndir)
    z = x[..., 0]
    rhob = np.exp(-z / H)
    pb = rhob * 1.0 * H
    w[..., v["rhob"]] = rhob
    w[..., v["bg0"] + 1] = B0
    w[..., v["eb"]] = pb / (gamma - 1.0) + 0.5 * B0 * B0
    cs = math.sqrt(gamma * H)
    if amp is None:
        amp = 1.0e-3 * cs
    if perturb is not None:
        add_modes(w, x, ndim, ndir, perturb, seed=seed, rho_scale=rhob)
    up = [amp, omega, 0.5, 0.5, sigma, z0, dz0]
    prm = make_params(gamma=gamma, nu=nu, grav=[-1.0, 0.0, 0.0], courantpar=courantpar,
                      typeadvance=typeadvance, user=USR_STRAT, userpar=up)
    nw = v["nw"]
    types = [["fixed"] * nw, ["cont"] * nw] + [["periodic"] * nw for _ in range(2 * (ndim - 1))]
    return Problem(f"strat{'x'.join(map(str, n))}", ndim, ndir, tuple(n), prm, x, w, types,
                   nsteps=nsteps, meta=dict(cs=cs, amp=amp))


def add_modes(w, x, ndim, ndir, amp, nmodes=64, kmax=16, seed=0, rho_scale=None):
    """Seeded random-phase Fourier modes (|k|<=kmax) added to rho', v and b'
    (divergence-free b' by projecting each mode's amplitude orthogonal to k).
    Momentum is set as (rho_b+rho') v.

    The grid is a tensor product of 1D axes, so each mode is a product of 1D
    complex exponentials; the sum over modes runs as one complex matrix product
    (planes of the first ndim-1 axes times the last axis), which keeps 512^3
    states within seconds."""
    rng = np.random.default_rng(seed)
    v = var_index(ndir)
    L = [x[..., d].max() - x[..., d].min() for d in range(ndim)]
    L = [l * (1 + 1.0 / (x.shape[d] - 1)) for d, l in enumerate(L)]
    axes = []
    for d in range(ndim):
        idx = [0] * ndim
        idx[d] = slice(None)
        axes.append(x[tuple(idx) + (d,)])
    ks, phs, avs, abs_ = [], [], [], []
    for _ in range(nmodes):
        while True:
            k = rng.integers(-kmax, kmax + 1, size=ndim)
            if 0 < np.linalg.norm(k) <= kmax:
                break
        ph = rng.uniform(0, 2 * math.pi, size=3)
        av = rng.normal(size=ndir)
        ab = rng.normal(size=ndir)
        kk = np.zeros(ndir)
        kk[:ndim] = k / np.asarray(L)
        ab = ab - kk * (ab @ kk) / (kk @ kk)
        ks.append(k)
        phs.append(ph)
        avs.append(av)
        abs_.append(ab)
    ks = np.array(ks)
    phs = np.array(phs)
    shape = x.shape[:-1]
    # E_d[m, i] = exp(i 2 pi k_d x_d / L_d)
    E = [np.exp(1j * 2 * math.pi * ks[:, d, None] * axes[d][None, :] / L[d]) for d in range(ndim)]
    lead = np.ones((nmodes, 1), dtype=complex)
    for d in range(ndim - 1):
        lead = (lead[:, :, None] * E[d][:, None, :]).reshape(nmodes, -1)
    last = E[ndim - 1]                                      # [m][n_last]

    def field(coef):  # sum_m Im(coef_m * e^{i phase_m}) on the grid
        out = (lead.T * coef[None, :]) @ last                # [(lead)][last]
        return np.imag(out).reshape(shape[:-1] + shape[-1:]) if ndim > 1 else np.imag(out).reshape(shape)

    drho = field(np.exp(1j * phs[:, 0]))
    dv = np.stack([field(np.exp(1j * phs[:, 1]) * np.array([a[c] for a in avs])) for c in range(ndir)], axis=-1)
    db = np.stack([field(np.exp(1j * phs[:, 2]) * np.array([a[c] for a in abs_])) for c in range(ndir)], axis=-1)
    norm = lambda a: a / max(np.abs(a).max(), 1e-300)  # noqa: E731
    drho = amp * norm(drho)
    dv = amp * norm(dv)
    db = amp * norm(db)
    rs = 1.0 if rho_scale is None else rho_scale
    w[..., v["rho"]] += drho * rs
    rt = w[..., v["rho"]] + w[..., v["rhob"]]
    for c in range(ndir):
        w[..., v["m0"] + 1 + c] += rt * dv[..., c]
        w[..., v["b0"] + 1 + c] += db[..., c]
    # keep the thermal pressure: e' gains kinetic and magnetic perturbation energy
    m2 = sum(w[..., v["m0"] + 1 + c] ** 2 for c in range(ndir))
    b2 = sum(w[..., v["b0"] + 1 + c] ** 2 for c in range(ndir))
    bb = sum(w[..., v["b0"] + 1 + c] * w[..., v["bg0"] + 1 + c] for c in range(ndir))
    w[..., v["e"]] += 0.5 * m2 / rt + 0.5 * b2 + bb


# ---------------------------------------------------------------------------
# generic randomised state for parity tests (every flux and source term active)
# ---------------------------------------------------------------------------
def random_problem(nx, ndir=None, seed=1, types=None, amp=0.05, gamma=5.0 / 3.0, nu=1.0,
                   grav=(-0.7, 0.3, 0.2), user=None, typeadvance="fourstep",
                   courantpar=0.4) -> Problem:
    ndim = len(nx)
    if ndir is None:
        ndir = max(ndim, 2) if ndim < 3 else 3
    rng = np.random.default_rng(seed)
    lows = tuple(0.1 * d for d in range(ndim))
    highs = tuple(1.0 + 0.25 * d for d in range(ndim))
    x = make_grid(nx, lows, highs)
    w = empty_state(nx, ndir)
    v = var_index(ndir)
    z = x[..., 0]
    w[..., v["rhob"]] = 1.0 + 0.5 * np.exp(-z)
    for c in range(ndir):
        w[..., v["bg0"] + 1 + c] = 0.3 - 0.1 * c + 0.05 * np.sin(1.0 + c + z)
    bg2 = sum(w[..., v["bg0"] + 1 + c] ** 2 for c in range(ndir))
    w[..., v["eb"]] = 0.8 * w[..., v["rhob"]] / (gamma - 1.0) + 0.5 * bg2
    add_modes(w, x, ndim, ndir, amp, nmodes=12, kmax=3, seed=seed)
    # a little white noise so that the hyperdiffusion windows see varied data
    for iw in range(v["eb"]):
        w[..., iw] += amp * 0.02 * rng.standard_normal(w.shape[:-1])
    if user is None:
        from .params import USR_GRAVVISC
        user = USR_GRAVVISC
    g = list(grav[:ndim]) + [0.0] * (3 - ndim)
    prm = make_params(gamma=gamma, nu=nu, grav=g, courantpar=courantpar, typeadvance=typeadvance,
                      user=user)
    nw = v["nw"]
    if types is None:
        types = ["cont"] * (2 * ndim)
    tl = [[t] * nw if isinstance(t, str) else list(t) for t in types]
    return Problem(f"random{'x'.join(map(str, nx))}", ndim, ndir, tuple(nx), prm, x, w, tl)


def orszag_tang(n=(64, 64), beta=1.0, gamma=5.0 / 3.0, B0=None, nu=1.0, typeadvance="fourstep",
                courantpar=0.8) -> Problem:
    """Orszag-Tang-type vortex on [0,1]^2, periodic: rho=gamma^2, v=(-sin2pi y,
    sin2pi x), B=B0(-sin2pi y, sin4pi x); p from the plasma beta 2p/<B^2>;
    zero background, everything carried as perturbation."""
    ndim, ndir = 2, 2
    x = make_grid(n, (0.0, 0.0), (1.0, 1.0))
    w = empty_state(n, ndir)
    v = var_index(ndir)
    X, Y = x[..., 0], x[..., 1]
    if B0 is None:
        B0 = 1.0
    rho = gamma ** 2 * np.ones_like(X)
    vx, vy = -np.sin(2 * math.pi * Y), np.sin(2 * math.pi * X)
    bx, by = B0 * -np.sin(2 * math.pi * Y), B0 * np.sin(4 * math.pi * X)
    bmean2 = B0 * B0  # <bx^2+by^2> = B0^2 (1/2 + 1/2)
    p = beta * bmean2 / 2.0
    w[..., v["rho"]] = rho
    w[..., v["m0"] + 1] = rho * vx
    w[..., v["m0"] + 2] = rho * vy
    w[..., v["b0"] + 1] = bx
    w[..., v["b0"] + 2] = by
    w[..., v["e"]] = p / (gamma - 1) + 0.5 * rho * (vx ** 2 + vy ** 2) + 0.5 * (bx ** 2 + by ** 2)
    # hyperdiffusion with the viscous dt limit (gravity module, zero gravity)
    from .params import USR_GRAVVISC
    prm = make_params(gamma=gamma, nu=nu, courantpar=courantpar, typeadvance=typeadvance, user=USR_GRAVVISC,
                      grav=(0.0, 0.0, 0.0))
    return Problem(f"ot{n[0]}x{n[1]}", ndim, ndir, tuple(n), prm, x, w,
                   uniform_types(ndim, v["nw"], "periodic"))


# ---------------------------------------------------------------------------
# 2D magnetic flux tube in a stratified atmosphere (x1 vertical, x2 horizontal)
# ---------------------------------------------------------------------------
def flux_tube(n=(256, 256), height=2.0, half_width=1.0, H=0.3, B0=0.5, tube_w2=0.04, g=1.0, rho0=100.0,
              gamma=5.0 / 3.0, A=1.0e-3, omega=None, z0=0.1, dz0=0.05, drv_w=0.1, nu=1.0,
              courantpar=0.8, dtpar=-1.0, typeadvance="fourstep") -> Problem:
    """Vertical flux tube B_b = (B_z(x), 0), B_z = B0 exp(-x^2/tube_w2), in an
    atmosphere with rho_b = rho0 exp(-z/H) and gravity g along -x1, on z in [0, height]
    (x1), x in [-half_width, half_width] (x2).

    Magnetohydrostatic balance is exact: with straight vertical field lines the
    Lorentz force is the horizontal magnetic-pressure gradient only, so
    p_b = rho0 g H exp(-z/H) + (B0^2 - B_z(x)^2)/2 balances it in x (p_b + B_z^2/2
    depends on z alone) and balances gravity in z (d p_b/dz = -rho_b g).  The
    gas is isothermal (p_b/rho_b = g H) on the tube axis; away from it the
    constant B0^2/2 added to the pressure heats the upper layers.  rho0 = 100
    puts the plasma-beta = 1 layer of the tube axis inside the domain (beta 240
    at the base, 0.3 at the top) and keeps the fastest wave speed near 1.6.  Zero
    initial perturbation; a horizontal velocity driver
    v_x = A sin(omega t) exp(-x^2/drv_w^2) exp(-(z-z0)^2/dz0^2) near the base
    (omega defaults to the acoustic cut-off sqrt(gamma g H)/(2H)); open (cont)
    x1 boundaries, periodic x2."""
    ndim, ndir = 2, 2
    x = make_grid(n, (0.0, -half_width), (height, half_width))
    w = empty_state(n, ndir)
    v = var_index(ndir)
    z, xh = x[..., 0], x[..., 1]
    rhob = rho0 * np.exp(-z / H)
    bz = B0 * np.exp(-(xh * xh) / tube_w2)
    pb = g * H * rhob + 0.5 * (B0 * B0 - bz * bz)
    w[..., v["rhob"]] = rhob
    w[..., v["bg0"] + 1] = bz
    w[..., v["eb"]] = pb / (gamma - 1.0) + 0.5 * bz * bz
    omega_ac = math.sqrt(gamma * g * H) / (2.0 * H)
    if omega is None:
        omega = omega_ac
    up = [A, omega, z0, dz0, 0.0, drv_w]
    prm = make_params(gamma=gamma, nu=nu, grav=[-g, 0.0, 0.0], courantpar=courantpar, dtpar=dtpar,
                      typeadvance=typeadvance, user=USR_TUBE, userpar=up)
    nw = v["nw"]
    types = [["cont"] * nw, ["cont"] * nw, ["periodic"] * nw, ["periodic"] * nw]
    return Problem(f"tube{n[0]}x{n[1]}", ndim, ndir, tuple(n), prm, x, w, types,
                   meta=dict(omega_ac=omega_ac, A=A, omega=omega))


__all__ = ["Problem", "brio_wu", "stratified", "random_problem", "orszag_tang", "flux_tube", "var_index",
           "USR_NONE", "USR_TUBE"]
