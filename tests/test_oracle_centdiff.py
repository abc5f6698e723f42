"""The oracle's flux divergence against a numpy transcription of the Fortran (CPU).

centdiff4 (src/vaccd.t:7-78) with getv (src/vacphys0.t.mhd), getflux
(src/vacphys.mhd0.t:147-222), getptotal / getptotal_bg (src/vacphys0.t.mhd) and
gradient4 (src/vacgrid.t:665-712), written here as whole-array statements in the
Fortran's evaluation order.  One 'cd4' step of typeadvance='onestep' with no
user module adds no source, so the oracle's mesh update must equal
w - dt * (flux divergence + the energy equation's background work) exactly."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import params, problems

import _util


def _mesh(P, a, d=None, k=0):
    sl = []
    for e in range(P.ndim):
        lo = 2 + (k if e == d else 0)
        sl.append(slice(lo, lo + P.nx[e]))
    return a[tuple(sl)]


def _gradient4(P, q, d):
    """gradient4 on the mesh: -(q(+2) - 8(q(+1) - q(-1)) - q(-2))/dx/12, the two
    edge layers along d zeroed."""
    x = P.x[..., d]
    dx = 0.5 * (_mesh(P, x, d, 1) - _mesh(P, x, d, -1))
    g = -(_mesh(P, q, d, 2) - 8.0 * (_mesh(P, q, d, 1) - _mesh(P, q, d, -1)) - _mesh(P, q, d, -2)) / dx / 12.0
    idx = [slice(None)] * P.ndim
    for layer in (0, 1, -1, -2):
        idx[d] = layer
        g[tuple(idx)] = 0.0
    return g


def _csum(terms):
    s = terms[0]
    for t in terms[1:]:
        s = s + t
    return s


def _getptotal(w, v, ndir, gamma):
    b = [w[..., v["b0"] + 1 + c] for c in range(ndir)]
    bg = [w[..., v["bg0"] + 1 + c] for c in range(ndir)]
    m = [w[..., v["m0"] + 1 + c] for c in range(ndir)]
    p = (gamma - 2.0) * (_csum([b[c] * bg[c] for c in range(ndir)]) + 0.5 * _csum([b[c] * b[c] for c in range(ndir)]))
    return (gamma - 1.0) * (w[..., v["e"]] - 0.5 * _csum([m[c] * m[c] for c in range(ndir)])
                            / (w[..., v["rho"]] + w[..., v["rhob"]])) - p


def _getptotal_bg(w, v, ndir, gamma):
    bg = [w[..., v["bg0"] + 1 + c] for c in range(ndir)]
    return (gamma - 1.0) * w[..., v["eb"]] - 0.5 * (gamma - 2.0) * _csum([bg[c] * bg[c] for c in range(ndir)])


def _getflux(w, v, ndir, gamma, iw, d):
    """getflux: the non-transported flux of iw along d, and whether the transport
    flux v_d w(iw) is added."""
    rt = w[..., v["rho"]] + w[..., v["rhob"]]
    m = [w[..., v["m0"] + 1 + c] for c in range(ndir)]
    b = [w[..., v["b0"] + 1 + c] for c in range(ndir)]
    bg = [w[..., v["bg0"] + 1 + c] for c in range(ndir)]
    if iw == v["rho"]:
        return w[..., v["rhob"]] * m[d] / rt, True
    if v["m0"] < iw <= v["m0"] + ndir:
        C = iw - v["m0"] - 1
        if C == d:
            f = _getptotal(w, v, ndir, gamma)
            fb = np.zeros_like(f)  # getptotal_bg, then fb=0 (perturbed form)
            return f + fb - (b[C] * bg[d] + b[d] * bg[C]) - b[C] * b[d], True
        return -(b[C] * bg[d] + b[d] * bg[C]) - b[C] * b[d], True
    if iw == v["e"]:
        f = _getptotal(w, v, ndir, gamma)
        fb = np.zeros_like(f)
        s1 = _csum([bg[c] * m[c] for c in range(ndir)])
        s2 = _csum([b[c] * m[c] for c in range(ndir)])
        return ((m[d] * (f + fb) - b[d] * s1 - bg[d] * s2) / rt + w[..., v["eb"]] * m[d] / rt
                - b[d] * s2 / rt), True
    C = iw - v["b0"] - 1
    if C == d:
        return np.zeros_like(rt), False
    return -(m[C] / rt * (b[d] + bg[d])) + m[d] / rt * bg[C], True


def _centdiff4(P, w, qdt, dims):
    """The mesh part of w after centdiff4 over the dimensions dims, from wCT = w."""
    v = problems.var_index(P.ndir)
    gamma = P.params.gamma
    new = _mesh(P, w).copy()
    for d in dims:
        vel = w[..., v["m0"] + 1 + d] / (w[..., v["rho"]] + w[..., v["rhob"]])  # getv
        for iw in range(v["eb"]):
            f, transport = _getflux(w, v, P.ndir, gamma, iw, d)
            if transport:
                f = f + vel * w[..., iw]
            new[..., iw] = new[..., iw] - qdt * _gradient4(P, f, d)
            if iw == v["e"]:
                fb = _mesh(P, _getptotal_bg(w, v, P.ndir, gamma))
                new[..., iw] = new[..., iw] - qdt * _gradient4(P, vel, d) * fb
                for di in dims:
                    bgi = _mesh(P, w[..., v["bg0"] + 1 + di])
                    bgd = _mesh(P, w[..., v["bg0"] + 1 + d])
                    new[..., iw] = new[..., iw] + qdt * bgi * bgd * _gradient4(P, vel, di)
    return new


@pytest.mark.parametrize("nx,ndir,split", [((30,), 2, None), ((30,), 3, None), ((14, 12), 2, None),
                                           ((14, 12), 3, None), ((14, 12), 3, 2), ((10, 9, 8), 3, None),
                                           ((10, 9, 8), 3, 1)])
def test_flux_divergence_step_matches_numpy(nx, ndir, split):
    types = ["cont", "fixed", "periodic", "periodic", "cont", "symm"][: 2 * len(nx)]
    P = problems.random_problem(nx, ndir=ndir, seed=37, types=types, user=params.USR_NONE, typeadvance="onestep")
    o = _util.start(Oracle, P)
    w0 = o.download()
    # a step far beyond stability, so that the increment dominates w and any
    # difference in the last bit of a flux shows in the result
    qdt = 37.0
    if split is None:
        o.advect(qdt, 0.0, 0)
        dims = list(range(len(nx)))
    else:
        o.advect(qdt, 0.0, 0, idimmin=split, idimmax=split)
        dims = [split - 1]
    got = _util.mesh(P, o.download())
    want = _centdiff4(P, w0, qdt, dims)
    nadv = 2 * P.ndir + 2
    assert np.abs(got[..., :nadv] - _util.mesh(P, w0)[..., :nadv]).max() > 1e-6  # the fluxes act
    np.testing.assert_array_equal(got[..., :nadv], want[..., :nadv])


def test_flux_divergence_for_random_shapes():
    """Hypothesis-drawn grids (1D-3D, 5 to 9 mesh cells per dimension), ndir and a
    split dimension: one cd4 step, bit for bit."""
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @settings(max_examples=20, deadline=None, derandomize=True)
    @given(st.lists(st.integers(5, 9), min_size=1, max_size=3), st.integers(0, 2 ** 16), st.booleans(),
           st.integers(0, 3))
    def check(nx, seed, ndir3, split):
        nd = len(nx)
        ndir = 3 if (ndir3 or nd == 3) else max(nd, 2)
        P = problems.random_problem(tuple(nx), ndir=ndir, seed=seed, types=["cont", "cont"] * nd,
                                    user=params.USR_NONE, typeadvance="onestep")
        o = _util.start(Oracle, P)
        w0 = o.download()
        if split == 0 or split > nd:
            o.advect(37.0, 0.0, 0)
            dims = list(range(nd))
        else:
            o.advect(37.0, 0.0, 0, idimmin=split, idimmax=split)
            dims = [split - 1]
        got = _util.mesh(P, o.download())
        o.close()
        nadv = 2 * P.ndir + 2
        np.testing.assert_array_equal(got[..., :nadv], _centdiff4(P, w0, 37.0, dims)[..., :nadv])

    check()
