"""The oracle's hyperdiffusion against a numpy transcription of the Fortran (CPU).

addsource_visc (src/vacusr.viscosity.t:2-221) with setnu (:223-450), the
zero-bodied setnushk, gradient1 / gradient1L / gradient1R (:547-675) and
getcmax / getcsound2 / getpthermal (src/vacphys0.t.mhd:77-186), written as
whole-array statements in the Fortran's loop and evaluation order.  nuL and nuR
are 0 outside the mesh, as the oracle and the CUDA path define them (the
reference leaves those entries of its local arrays unset).

One 'source' step of typeadvance='onestep' with the gravity/viscosity module and
zero gravity adds only this source, so the oracle's mesh update must equal
w + addsource_visc(w) exactly."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import params, problems

import _util


def _reg(P, a, g=0, d=None, k=0):
    """a on the mesh grown by g layers, shifted by k cells along d."""
    sl = []
    for e in range(P.ndim):
        lo = 2 - g + (k if e == d else 0)
        sl.append(slice(lo, lo + P.nx[e] + 2 * g))
    return a[tuple(sl)]


class Visc:
    def __init__(self, P, w, qdt):
        self.P, self.w, self.qdt = P, w, qdt
        self.v = problems.var_index(P.ndir)
        self.gamma = P.params.gamma
        self.rt = w[..., self.v["rho"]] + w[..., self.v["rhob"]]
        # gradient1* zero the two edge layers of their range (the mesh grown by
        # one) along d unless rho's boundary there is periodic
        self.periodic = [[P.typeB[2 * d + s][0] == "periodic" for s in (0, 1)] for d in range(P.ndim)]
        self.dxg = _util.gridsetup1_dx(P)
        self.maxviscoef = 0.0

    # ---- grid helpers --------------------------------------------------------
    def dx(self, g, d):
        return _reg(self.P, self.dxg[..., d], g)

    def zero_edges(self, a, d):
        idx = [slice(None)] * self.P.ndim
        if not self.periodic[d][0]:
            for layer in (0, 1):
                idx[d] = layer
                a[tuple(idx)] = 0.0
        if not self.periodic[d][1]:
            for layer in (-1, -2):
                idx[d] = layer
                a[tuple(idx)] = 0.0
        return a

    def gradient1L(self, q, d):  # on the mesh grown by one, q on the full grid
        P = self.P
        return self.zero_edges((_reg(P, q, 1) - _reg(P, q, 1, d, -1)) / self.dx(1, d), d)

    def gradient1R(self, q, d):
        P = self.P
        return self.zero_edges((_reg(P, q, 1, d, 1) - _reg(P, q, 1)) / self.dx(1, d), d)

    def gradient1_r1(self, q1, d):
        """gradient1 of q1 given on the mesh grown by one, on the mesh."""
        P = self.P
        sl = lambda k: tuple(slice(1 + (k if e == d else 0), 1 + (k if e == d else 0) + P.nx[e])  # noqa: E731
                             for e in range(P.ndim))
        g = (q1[sl(1)] - q1[sl(-1)]) / self.dx(0, d) / 2.0
        idx = [slice(None)] * P.ndim  # the zeroed layers of the grown range that lie on the mesh
        if not self.periodic[d][0]:
            idx[d] = 0
            g[tuple(idx)] = 0.0
        if not self.periodic[d][1]:
            idx[d] = -1
            g[tuple(idx)] = 0.0
        return g

    def gradient1(self, q, d):
        P = self.P
        return self.zero_edges((_reg(P, q, 1, d, 1) - _reg(P, q, 1, d, -1)) / self.dx(1, d) / 2.0, d)

    # ---- physics -------------------------------------------------------------
    def csum(self, terms):
        s = terms[0]
        for t in terms[1:]:
            s = s + t
        return s

    def cmax(self, d):
        """getcmax along d on the full grid (getcsound2, getpthermal)."""
        w, v, g, nd = self.w, self.v, self.gamma, self.P.ndir
        m = [w[..., v["m0"] + 1 + c] for c in range(nd)]
        b = [w[..., v["b0"] + 1 + c] for c in range(nd)]
        bg = [w[..., v["bg0"] + 1 + c] for c in range(nd)]
        rt = self.rt
        p = 0.5 * self.csum([x * x for x in m]) / rt
        p = p + 0.5 * self.csum([x * x for x in b]) + self.csum([b[c] * bg[c] for c in range(nd)])
        p = (g - 1.0) * (w[..., v["e"]] - p)
        cs2 = g * (p + (g - 1.0) * (w[..., v["eb"]] - 0.5 * self.csum([x * x for x in bg]))) / rt
        cf2 = self.csum([(b[c] + bg[c]) * (b[c] + bg[c]) for c in range(nd)]) / rt + cs2
        Bd = b[d] + bg[d]
        return np.sqrt(0.5 * (cf2 + np.sqrt(cf2 * cf2 - 4.0 * cs2 * (Bd * Bd) / rt))) + np.abs(m[d] / rt)

    def q173(self):
        w, v, nd = self.w, self.v, self.P.ndir
        b2 = self.csum([w[..., v["b0"] + 1 + c] * w[..., v["b0"] + 1 + c] for c in range(nd)])
        m2 = self.csum([w[..., v["m0"] + 1 + c] * w[..., v["m0"] + 1 + c] for c in range(nd)])
        return w[..., v["e"]] - 0.5 * (b2 + m2 / self.rt)

    def setnu(self, q, chyp, d):
        """nuR, nuL on the mesh grown by one (0 outside the mesh)."""
        P = self.P
        c_tot = _reg(P, self.cmax(d)).max()
        n = P.nx[d]
        # tmp_nuI: one more layer along d, the mirror of mesh cell lo+3 / hi-3
        lo_m = np.take(q, [2 + 3], axis=d)
        hi_m = np.take(q, [n + 1 - 3], axis=d)
        t = np.concatenate([lo_m, q, hi_m], axis=d)  # full-grid index i -> i + 1

        def T(i):  # t at full-grid positions i (an index array along d), the others on the mesh
            sl = []
            for e in range(P.ndim):
                if e == d:
                    sl.append(i)
                else:
                    sl.append(slice(2, 2 + P.nx[e]))
            return t[tuple(sl)]

        mesh = np.arange(2, 2 + n) + 1  # t-index of the mesh cells along d
        def d1R(f):  # |q(f+1) - q(f)|, f a t-index  # noqa: E306
            return np.abs(T(f + 1) - T(f))

        def d3R(f):
            return np.abs(3.0 * (T(f + 1) - T(f)) - (T(f + 2) - T(f - 1)))

        def d1L(f):
            return np.abs(T(f) - T(f - 1))

        def d3L(f):
            return np.abs(3.0 * (T(f) - T(f - 1)) - (T(f + 1) - T(f - 2)))

        md3R = np.maximum(np.maximum(d3R(mesh - 1), d3R(mesh)), d3R(mesh + 1))
        md1R = d1R(mesh - 2)
        for o in (-1, 0, 1, 2):
            md1R = np.maximum(md1R, d1R(mesh + o))
        md3L = np.maximum(np.maximum(d3L(mesh - 1), d3L(mesh)), d3L(mesh + 1))
        md1L = d1L(mesh - 2)
        for o in (-1, 0, 1, 2):
            md1L = np.maximum(md1L, d1L(mesh + o))
        dxm = self.dx(0, d)
        with np.errstate(divide="ignore", invalid="ignore"):
            nuR = np.where(md1R > 0.0, c_tot * chyp * md3R / md1R * dxm, 0.0)
            nuL = np.where(md1L > 0.0, c_tot * chyp * md3L / md1L * dxm, 0.0)
        # maxviscoef=MAX(MAXVAL(nuR), maxviscoef), then the same for nuL (:426, :444)
        self.maxviscoef = max(float(nuR.max()), self.maxviscoef)
        self.maxviscoef = max(float(nuL.max()), self.maxviscoef)
        R, L = np.zeros([x + 2 for x in P.nx]), np.zeros([x + 2 for x in P.nx])
        inner = tuple(slice(1, 1 + x) for x in P.nx)
        R[inner], L[inner] = nuR, nuL
        return R, L

    # ---- addsource_visc --------------------------------------------------------
    def step(self, base=None):
        """The mesh of base (default: w itself) plus addsource_visc of w."""
        P, w, v, qdt = self.P, self.w, self.v, self.qdt
        nd = P.ndim
        new = (_reg(P, w) if base is None else base).copy()
        inner = tuple(slice(1, 1 + x) for x in P.nx)
        nushk = 0.0
        # density and the "173" energy, :45-64
        for iw, q, chyp in ((v["rho"], w[..., v["rho"]], 0.04), (v["e"], self.q173(), 0.04)):
            for d in range(nd):
                nuR, nuL = self.setnu(q, chyp, d)
                tL = (nuL + nushk) * self.gradient1L(q, d)
                tR = (nuR + nushk) * self.gradient1R(q, d)
                new[..., iw] = new[..., iw] + (tR - tL)[inner] / self.dx(0, d) * qdt
        # momentum, :69-133
        rtC = self.rt
        for k in range(nd):
            rL = ((_reg(P, rtC)) + (_reg(P, rtC, 0, k, -1))) / 2.0
            rR = ((_reg(P, rtC, 0, k, 1)) + (_reg(P, rtC))) / 2.0
            for l in range(nd):
                q = w[..., v["m0"] + 1 + l] / self.rt
                nuR, nuL = self.setnu(q, 0.4, k)
                for ii1 in (0, 1):
                    i, ii0 = (k, l) if ii1 == 0 else (l, k)
                    m = w[..., v["m0"] + 1 + ii0]
                    if i == k:
                        VL = (_reg(P, m) + _reg(P, m, 0, k, -1)) / 2.0
                        VR = (_reg(P, m, 0, k, 1) + _reg(P, m)) / 2.0
                        tL = ((nuL + nushk) * self.gradient1L(q, k))[inner]
                        tR = ((nuR + nushk) * self.gradient1R(q, k))[inner]
                        t2 = (rR * tR - rL * tL) / self.dx(0, k) / 2.0
                        new[..., v["m0"] + 1 + ii0] = new[..., v["m0"] + 1 + ii0] + t2 * qdt
                        t2 = (VR * tR - VL * tL) / self.dx(0, k) / 2.0
                        new[..., v["e"]] = new[..., v["e"]] + t2 * qdt
                    else:
                        t2 = self.gradient1(q, k) * (nuL + nuR + 2.0 * nushk) / 2.0 / 2.0
                        tC = self.gradient1_r1(_reg(P, rtC, 1) * t2, i)
                        new[..., v["m0"] + 1 + ii0] = new[..., v["m0"] + 1 + ii0] + tC * qdt
                        tC = self.gradient1_r1(_reg(P, m, 1) * t2, i)
                        new[..., v["e"]] = new[..., v["e"]] + tC * qdt
        # magnetic field, :139-215 (no field diffusion in 1D: k != l never holds)
        for k in range(nd):
            for l in range(nd):
                if k == l:
                    continue
                b = w[..., v["b0"] + 1 + l]
                nuR, nuL = self.setnu(b, 0.04, k)
                for ii1 in (0, 1):
                    if ii1 == 0:
                        ii0, mm, sB, j = k, l, -1.0, k
                    else:
                        ii0, mm, sB, j = l, k, 1.0, l
                    bj = w[..., v["b0"] + 1 + j]
                    if mm == k:
                        BL = (_reg(P, bj) + _reg(P, bj, 0, mm, -1)) / 2.0
                        BR = (_reg(P, bj, 0, mm, 1) + _reg(P, bj)) / 2.0
                        tL = (nuL * self.gradient1L(b, k))[inner]
                        tR = (nuR * self.gradient1R(b, k))[inner]
                        new[..., v["b0"] + 1 + ii0] = (new[..., v["b0"] + 1 + ii0]
                                                       + sB * (tR - tL) / self.dx(0, k) * qdt)
                        new[..., v["e"]] = new[..., v["e"]] + sB * (tR * BR - tL * BL) / self.dx(0, k) * qdt
                    else:
                        t2 = self.gradient1(b, k) * (nuL + nuR) / 2.0
                        tC = self.gradient1_r1(t2, mm)
                        new[..., v["b0"] + 1 + ii0] = new[..., v["b0"] + 1 + ii0] + sB * tC * qdt
                        t2 = t2 * _reg(P, bj, 1)
                        tC = self.gradient1_r1(t2, mm)
                        new[..., v["e"]] = new[..., v["e"]] + sB * tC * qdt
        return new


@pytest.mark.parametrize("nx,ndir,types", [
    ((30,), 2, ["cont", "symm"]),
    ((30,), 3, ["periodic", "periodic"]),
    ((14, 12), 2, ["cont", "fixed", "periodic", "periodic"]),
    ((14, 12), 3, ["periodic", "periodic", "cont", "cont"]),
    ((10, 9, 8), 3, ["cont", "fixed", "periodic", "periodic", "cont", "symm"]),
])
def test_hyperdiffusion_step_matches_numpy(nx, ndir, types):
    P = problems.random_problem(nx, ndir=ndir, seed=38, types=types, user=params.USR_GRAVVISC,
                                grav=(0.0, 0.0, 0.0), typeadvance="onestep")
    o = _util.start(Oracle, P)
    w0 = o.download()
    qdt = 37.0  # the increment dominates w, so its last bits show
    o.advect(qdt, 0.0, 0, method="source")
    got = _util.mesh(P, o.download())
    want = Visc(P, w0, qdt).step()
    nadv = 2 * P.ndir + 2
    assert np.abs(got[..., :nadv] - _util.mesh(P, w0)[..., :nadv]).max() > 1e-6  # the source acts
    np.testing.assert_array_equal(got[..., :nadv], want[..., :nadv])


@pytest.mark.parametrize("nx,ndir", [((30,), 2), ((14, 12), 3), ((10, 9, 8), 3)])
def test_first_dt_matches_numpy(nx, ndir):
    """getdt at the first step (src/vac.t:61-70): getdt_courant (src/vac.t:641-699),
    getdt_visc with maxviscoef still 0 (an infinite limit), and getdt_grav, whose
    limit takes every gravity component over the cell widths of every dimension
    (src/vacusr.gravity.t:97-138)."""
    types = ["cont", "fixed", "periodic", "periodic", "cont", "symm"][: 2 * len(nx)]
    grav = (-0.7, 0.3, 0.2)
    P = problems.random_problem(nx, ndir=ndir, seed=40, types=types, user=params.USR_GRAVVISC, grav=grav)
    o = _util.start(Oracle, P)
    dt = o.getdt(0)
    V = Visc(P, o.download(), 0.0)
    courantmax = 0.0
    for d in range(P.ndim):
        courantmax = max(courantmax, float((_reg(P, V.cmax(d)) / V.dx(0, d)).max()))
    want = 1.0e99
    want = min(want, P.params.courantpar / courantmax)
    dtgrav = 1.0e99
    for d in range(P.ndim):
        m = max(float((abs(grav[d]) / V.dx(0, j)).max()) for j in range(P.ndim))
        dtgrav = min(dtgrav, 1.0 / np.sqrt(m))
    want = min(want, dtgrav)
    assert dt == want


def test_hyperdiffusion_for_random_shapes():
    """Hypothesis-drawn grids (1D-3D, 5 to 9 mesh cells per dimension), ndir and
    periodic dimensions: one hyperdiffusion step, bit for bit."""
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @settings(max_examples=20, deadline=None, derandomize=True)
    @given(st.lists(st.integers(5, 9), min_size=1, max_size=3), st.integers(0, 7), st.integers(0, 2 ** 16),
           st.booleans())
    def check(nx, periodic_mask, seed, ndir3):
        nd = len(nx)
        ndir = 3 if (ndir3 or nd == 3) else max(nd, 2)
        types = []
        for d in range(nd):
            types += ["periodic", "periodic"] if (periodic_mask >> d) & 1 else ["cont", "symm"]
        P = problems.random_problem(tuple(nx), ndir=ndir, seed=seed, types=types, user=params.USR_GRAVVISC,
                                    grav=(0.0, 0.0, 0.0), typeadvance="onestep")
        o = _util.start(Oracle, P)
        w0 = o.download()
        o.advect(37.0, 0.0, 0, method="source")
        got = _util.mesh(P, o.download())
        o.close()
        nadv = 2 * P.ndir + 2
        np.testing.assert_array_equal(got[..., :nadv], Visc(P, w0, 37.0).step()[..., :nadv])

    check()
