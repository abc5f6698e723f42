"""The oracle's optional source terms against direct numpy restatements (CPU).

Powell's div B source (addsource_divb, src/vacphys.mhd0.t:263-297) and the
resistive source (addsource_res2, src/vacphys.mhdres.t:231-301, and its compact
form addsource_res1, :96-220, both for a constant eta) are checked on one 'source' step of typeadvance='onestep' with no user module,
where the mesh update is exactly w_new = w + qdt S(w).  The Powell term is also
checked to be compiled out of 1D runs ({^NOONED}, src/vacphys.mhd0.t:255), and
the resistive dt limit (getdt_res, src/vacphys.mhdres.t:5-45) by its formula."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import params, problems

import _util


def _view(P, a, d=None, k=0):
    """a (full grid, first ndim axes) on the mesh shifted by k cells along d."""
    sl = []
    for e in range(P.ndim):
        lo = 2 + (k if e == d else 0)
        sl.append(slice(lo, lo + P.nx[e]))
    return a[tuple(sl)]


def _dx(P, d):
    x = P.x[..., d]
    return 0.5 * (_view(P, x, d, 1) - _view(P, x, d, -1))


def _gradient4(P, q, d):
    """gradient4 on the mesh, its two edge layers zeroed (src/vacgrid.t:665-712)."""
    g = -(_view(P, q, d, 2) - 8.0 * (_view(P, q, d, 1) - _view(P, q, d, -1)) - _view(P, q, d, -2)) / _dx(P, d) / 12.0
    idx = [slice(None)] * P.ndim
    for layer in (0, 1, -1, -2):
        idx[d] = layer
        g[tuple(idx)] = 0.0
    return g


def _powell_step(P, w, qdt, new=None):
    """The mesh after Powell's source from w added to new (default: w's mesh)."""
    v = problems.var_index(P.ndir)
    B = [w[..., v["b0"] + 1 + c] + w[..., v["bg0"] + 1 + c] for c in range(P.ndir)]
    divb = np.zeros(P.nx)
    for d in range(P.ndim):
        divb = divb + _gradient4(P, B[d], d)
    divb = qdt * divb
    rt = _view(P, w[..., v["rho"]] + w[..., v["rhob"]])
    new = _view(P, w).copy() if new is None else new.copy()
    s = 0.0
    for c in range(P.ndir):
        Bc = _view(P, B[c])
        mc = _view(P, w[..., v["m0"] + 1 + c])
        new[..., v["m0"] + 1 + c] = new[..., v["m0"] + 1 + c] - Bc * divb
        new[..., v["b0"] + 1 + c] = new[..., v["b0"] + 1 + c] - mc / rt * divb
        s = mc * Bc if c == 0 else s + mc * Bc
    new[..., v["e"]] = new[..., v["e"]] - s / rt * divb
    return new


@pytest.mark.parametrize("nx,ndir", [((14, 12), 2), ((14, 12), 3), ((10, 9, 8), 3)])
def test_powell_source_step_matches_numpy(nx, ndir):
    types = ["cont", "fixed", "periodic", "periodic", "cont", "symm"][: 2 * len(nx)]
    P = problems.random_problem(nx, ndir=ndir, seed=31, types=types, user=params.USR_NONE,
                                typeadvance="onestep")
    P.params.divbfix = 1
    o = _util.start(Oracle, P)
    w0 = o.download()
    qdt = 37.0  # the increment dominates w, so its last bits show
    o.advect(qdt, 0.0, 0, method="source")
    got = _util.mesh(P, o.download())
    want = _powell_step(P, w0, qdt)
    nadv = 2 * P.ndir + 2
    assert np.abs(got[..., :nadv] - _util.mesh(P, w0)[..., :nadv]).max() > 1e-6  # the source acts
    np.testing.assert_array_equal(got[..., :nadv], want[..., :nadv])


def test_powell_source_for_random_shapes():
    """Hypothesis-drawn 2D/3D grids (5 to 9 mesh cells per dimension), ndir and
    boundary types: one 'source' step with divbfix, bit for bit."""
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @settings(max_examples=15, deadline=None, derandomize=True)
    @given(st.lists(st.integers(5, 9), min_size=2, max_size=3), st.integers(0, 2 ** 16), st.booleans(),
           st.sampled_from(["cont", "fixed", "symm", "cont1"]))
    def check(nx, seed, ndir3, edge):
        nd = len(nx)
        types = [t for d in range(nd) for t in (("periodic", "periodic") if d == 1 else ("cont", edge))]
        P = problems.random_problem(tuple(nx), ndir=3 if (ndir3 or nd == 3) else 2, seed=seed, types=types,
                                    user=params.USR_NONE, typeadvance="onestep")
        P.params.divbfix = 1
        o = _util.start(Oracle, P)
        w0 = o.download()
        o.advect(37.0, 0.0, 0, method="source")
        got = _util.mesh(P, o.download())
        o.close()
        nadv = 2 * P.ndir + 2
        np.testing.assert_array_equal(got[..., :nadv], _powell_step(P, w0, 37.0)[..., :nadv])

    check()


def test_powell_source_is_off_in_1d():
    P = problems.random_problem((40,), ndir=3, seed=32)
    a = _util.start(Oracle, P)
    _util.run(a, 10)
    P.params.divbfix = 1
    b = _util.start(Oracle, P)
    _util.run(b, 10)
    np.testing.assert_array_equal(a.download(), b.download())


def test_powell_source_changes_a_2d_run():
    P = problems.random_problem((14, 12), seed=33, types=["cont", "cont", "periodic", "periodic"])
    a = _util.start(Oracle, P)
    _util.run(a, 5)
    P.params.divbfix = 1
    b = _util.start(Oracle, P)
    _util.run(b, 5)
    assert np.abs(a.download() - b.download()).max() > 1e-8


# ---------------------------------------------------------------------------
# resistivity
# ---------------------------------------------------------------------------
def _lvc(i, j, k):
    if i == j or j == k or i == k:
        return 0
    return 1 if (i + 1) % 3 == j else -1


def _region(P, a, g, d=None, k=0):
    """a on the mesh grown by g layers, shifted by k cells along d."""
    sl = []
    for e in range(P.ndim):
        lo = 2 - g + (k if e == d else 0)
        sl.append(slice(lo, lo + P.nx[e] + 2 * g))
    return a[tuple(sl)]


def _inner(P, T, d=None, k=0):
    """T given on the mesh grown by one layer: its mesh part shifted by k along d."""
    sl = []
    for e in range(P.ndim):
        lo = 1 + (k if e == d else 0)
        sl.append(slice(lo, lo + P.nx[e]))
    return T[tuple(sl)]


def _resist_step(P, w, qdt, eta, new=None):
    """The mesh after addsource_res2 from w added to new (default: w's mesh)."""
    v = problems.var_index(P.ndir)
    B = [w[..., v["b0"] + 1 + c] + w[..., v["bg0"] + 1 + c] for c in range(P.ndir)]
    dxg = _util.gridsetup1_dx(P)

    def dx(d, g):
        return _region(P, dxg[..., d], g)

    # J = curl B by the resistive module's gradient -(q(+1)-q(-1))/dx/2
    k0 = 6 - 2 * P.ndir
    J, idirmin = {}, 3
    for i in range(max(k0, 0), 3):
        J[i] = np.zeros([n + 2 for n in P.nx])
        for j in range(P.ndim):
            for k in range(P.ndir):
                sgn = _lvc(i, j, k)
                if sgn:
                    gr = -(_region(P, B[k], 1, j, 1) - _region(P, B[k], 1, j, -1)) / dx(j, 1) / 2.0
                    J[i] = J[i] + gr if sgn == 1 else J[i] - gr
                    idirmin = min(idirmin, i)
    new = _view(P, w).copy() if new is None else new.copy()

    def grad_mesh(T, d):
        return -(_inner(P, T, d, 1) - _inner(P, T, d, -1)) / dx(d, 0) / 2.0

    for i in range(P.ndir):
        iw = v["b0"] + 1 + i
        for j in range(P.ndim):
            for k in range(idirmin, 3):
                sgn = _lvc(i, j, k)
                if sgn:
                    t2 = grad_mesh(J[k] * eta * qdt, j)
                    new[..., iw] = new[..., iw] - t2 if sgn == 1 else new[..., iw] + t2
    for i in range(P.ndim):
        for j in range(P.ndir):
            for k in range(idirmin, 3):
                sgn = _lvc(i, j, k)
                if sgn:
                    t2 = grad_mesh(_region(P, B[j], 1) * J[k] * eta * qdt, i)
                    new[..., v["e"]] = new[..., v["e"]] + t2 if sgn == 1 else new[..., v["e"]] - t2
    return new


@pytest.mark.parametrize("nx,ndir", [((30,), 2), ((30,), 3), ((14, 12), 2), ((14, 12), 3), ((10, 9, 8), 3)])
def test_resistive_source_step_matches_numpy(nx, ndir):
    types = ["cont", "fixed", "periodic", "periodic", "cont", "symm"][: 2 * len(nx)]
    P = problems.random_problem(nx, ndir=ndir, seed=34, types=types, user=params.USR_NONE,
                                typeadvance="onestep")
    eta = 0.02
    P.params.eta = eta
    o = _util.start(Oracle, P)
    w0 = o.download()
    qdt = 37.0  # the increment dominates w, so its last bits show
    o.advect(qdt, 0.0, 0, method="source")
    got = _util.mesh(P, o.download())
    want = _resist_step(P, w0, qdt, eta)
    nadv = 2 * P.ndir + 2
    assert np.abs(got[..., :nadv] - _util.mesh(P, w0)[..., :nadv]).max() > 1e-6  # the source acts
    np.testing.assert_array_equal(got[..., :nadv], want[..., :nadv])


def _resist1_step(P, w, qdt, eta, new=None):
    """addsource_res1 (compactres=T, src/vacphys.mhdres.t:96-220) on the mesh:
    per idir, eta times the 3-point Laplacian of B_idir into b_idir and, times
    B_idir, into e; then eta J**2 into e, J from getcurrent on the mesh."""
    v = problems.var_index(P.ndir)
    B = [w[..., v["b0"] + 1 + c] + w[..., v["bg0"] + 1 + c] for c in range(P.ndir)]
    dxg = _util.gridsetup1_dx(P)
    k0 = 6 - 2 * P.ndir
    J, idirmin = {}, 3
    for i in range(max(k0, 0), 3):
        J[i] = np.zeros(P.nx)
        for j in range(P.ndim):
            for k in range(P.ndir):
                sgn = _lvc(i, j, k)
                if sgn:
                    gr = -(_view(P, B[k], j, 1) - _view(P, B[k], j, -1)) / _view(P, dxg[..., j]) / 2.0
                    J[i] = J[i] + gr if sgn == 1 else J[i] - gr
                    idirmin = min(idirmin, i)
    new = _view(P, w).copy() if new is None else new.copy()
    for i in range(P.ndir):
        tmp = np.zeros(P.nx)
        for d in range(P.ndim):
            dx = _view(P, dxg[..., d])
            tmp = tmp + (_view(P, B[i], d, 1) - 2 * _view(P, B[i]) + _view(P, B[i], d, -1)) / (dx * dx)
        tmp = tmp * eta
        new[..., v["b0"] + 1 + i] = new[..., v["b0"] + 1 + i] + qdt * tmp
        new[..., v["e"]] = new[..., v["e"]] + qdt * tmp * _view(P, B[i])
    j2 = np.zeros(P.nx)
    for i in range(idirmin, 3):
        j2 = j2 + J[i] * J[i]
    new[..., v["e"]] = new[..., v["e"]] + qdt * eta * j2
    return new


@pytest.mark.parametrize("nx,ndir", [((30,), 1), ((30,), 2), ((30,), 3), ((14, 12), 2), ((14, 12), 3),
                                     ((10, 9, 8), 3)])
def test_compact_resistive_source_step_matches_numpy(nx, ndir):
    types = ["cont", "fixed", "periodic", "periodic", "cont", "symm"][: 2 * len(nx)]
    P = problems.random_problem(nx, ndir=ndir, seed=37, types=types, user=params.USR_NONE,
                                typeadvance="onestep")
    eta = 0.02
    P.params.eta = eta
    P.params.compactres = 1
    o = _util.start(Oracle, P)
    w0 = o.download()
    qdt = 37.0
    o.advect(qdt, 0.0, 0, method="source")
    got = _util.mesh(P, o.download())
    want = _resist1_step(P, w0, qdt, eta)
    nadv = 2 * P.ndir + 2
    assert np.abs(got[..., :nadv] - _util.mesh(P, w0)[..., :nadv]).max() > 1e-6
    np.testing.assert_array_equal(got[..., :nadv], want[..., :nadv])
    # the two forms differ (the compact one is not conservative)
    P.params.compactres = 0
    o2 = _util.start(Oracle, P)
    o2.advect(qdt, 0.0, 0, method="source")
    assert np.abs(_util.mesh(P, o2.download())[..., :nadv] - got[..., :nadv]).max() > 1e-9


def test_resistive_sources_for_random_shapes():
    """Hypothesis-drawn grids (1D-3D, 5 to 9 mesh cells per dimension), ndir, eta
    and the form (compactres or not): one 'source' step, bit for bit."""
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @settings(max_examples=20, deadline=None, derandomize=True)
    @given(st.lists(st.integers(5, 9), min_size=1, max_size=3), st.integers(0, 2 ** 16), st.integers(1, 3),
           st.sampled_from([0.003, 0.02, 0.4]), st.booleans())
    def check(nx, seed, ndir, eta, compact):
        nd = len(nx)
        ndir = max(ndir, nd)
        types = [t for d in range(nd) for t in (("periodic", "periodic") if d == 0 else ("cont", "fixed"))]
        P = problems.random_problem(tuple(nx), ndir=ndir, seed=seed, types=types, user=params.USR_NONE,
                                    typeadvance="onestep")
        P.params.eta = eta
        P.params.compactres = int(compact)
        o = _util.start(Oracle, P)
        w0 = o.download()
        o.advect(37.0, 0.0, 0, method="source")
        got = _util.mesh(P, o.download())
        o.close()
        want = (_resist1_step if compact else _resist_step)(P, w0, 37.0, eta)
        nadv = 2 * P.ndir + 2
        np.testing.assert_array_equal(got[..., :nadv], want[..., :nadv])

    check()


def test_resistive_dt_limit():
    P = problems.random_problem((14, 12), seed=35, types=["cont", "cont", "periodic", "periodic"],
                                user=params.USR_NONE)
    o = _util.start(Oracle, P)
    dt0 = o.getdt(0)
    P.params.eta = 0.5
    o = _util.start(Oracle, P)
    dt1 = o.getdt(0)
    x = P.x
    mn = min(float((0.5 * (_view(P, x[..., d], d, 1) - _view(P, x[..., d], d, -1))).min()) for d in range(P.ndim))
    want = min(dt0, P.params.dtdiffpar * mn * mn / 0.5)
    assert want < dt0  # the diffusion limit decides
    np.testing.assert_allclose(dt1, want, rtol=1e-14)


def test_negative_eta_is_rejected():
    from sac_b200 import abi
    P = problems.random_problem((14, 12), seed=36, types=["cont", "cont", "periodic", "periodic"])
    P.params.eta = -0.1
    o = _util.start(Oracle, P)
    with pytest.raises(abi.SacError):
        o.getdt(0)
    with pytest.raises(abi.SacError):
        o.advect(0.01, 0.0, 0)


# ---------------------------------------------------------------------------
# gravity, addsource_grav (src/vacusr.gravity.t:24-81)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("nx,ndir", [((30,), 2), ((14, 12), 3), ((10, 9, 8), 3)])
def test_gravity_source_step_matches_numpy(nx, ndir):
    types = ["cont", "fixed", "periodic", "periodic", "cont", "symm"][: 2 * len(nx)]
    grav = (-0.7, 0.3, 0.2)
    P = problems.random_problem(nx, ndir=ndir, seed=39, types=types, user=params.USR_GRAVVISC, nu=0.0,
                                grav=grav, typeadvance="onestep")
    o = _util.start(Oracle, P)
    w0 = o.download()
    qdt = 37.0  # the increment dominates w, so its last bits show
    o.advect(qdt, 0.0, 0, method="source")
    got = _util.mesh(P, o.download())
    v = problems.var_index(P.ndir)
    want = _view(P, w0).copy()
    rho = _view(P, w0[..., v["rho"]])
    rt = _view(P, w0[..., v["rho"]] + w0[..., v["rhob"]])
    for d in range(P.ndim):  # dm_i/dt = +g_i rho' (the perturbed density only)
        want[..., v["m0"] + 1 + d] = want[..., v["m0"] + 1 + d] + qdt * grav[d] * rho
    for d in range(P.ndim):  # de/dt = +g_i rho' m_i/(rho'+rho_b)
        want[..., v["e"]] = want[..., v["e"]] + qdt * grav[d] * rho * _view(P, w0[..., v["m0"] + 1 + d]) / rt
    nadv = 2 * P.ndir + 2
    np.testing.assert_array_equal(got[..., :nadv], want[..., :nadv])


# ---------------------------------------------------------------------------
# the reference's Slog user module, specialsource (src/vacusr.f:1255-1382):
# gravity, hyperdiffusion (eqpar(nu_)=1), then the vortex velocity driver
# ---------------------------------------------------------------------------
def test_slog_source_step_matches_its_fortran():
    import math

    from test_oracle_visc import Visc

    P = problems.random_problem((10, 8, 8), seed=43, user=params.USR_SLOG,
                                types=["cont", "cont", "periodic", "periodic", "periodic", "periodic"],
                                typeadvance="onestep")
    P.x[...] *= 1.0e6  # the module's lengths are in metres (Mm scale), x1 vertical
    o = _util.start(Oracle, P)
    w0 = o.download()
    qdt, qt = 37.0, 30.0
    o.advect(qdt, qt, 0, method="source")
    got = _util.mesh(P, o.download())

    v = problems.var_index(P.ndir)
    new = _view(P, w0).copy()
    grav = list(P.params.grav)
    rho = _view(P, w0[..., v["rho"]])
    rt = _view(P, w0[..., v["rho"]] + w0[..., v["rhob"]])
    for d in range(3):
        if abs(grav[d]) > 1e-99:
            new[..., v["m0"] + 1 + d] = new[..., v["m0"] + 1 + d] + qdt * grav[d] * rho
    for d in range(3):
        if abs(grav[d]) > 1e-99:
            new[..., v["e"]] = new[..., v["e"]] + qdt * grav[d] * rho * _view(P, w0[..., v["m0"] + 1 + d]) / rt
    new = Visc(P, w0, qdt).step(new)
    # the driver, with the single-precision literals pi, 0.1 and 0.05, and the
    # density already updated by the hyperdiffusion
    f32 = lambda a: float(np.float32(a))  # noqa: E731
    pi = f32(math.pi)
    xc1, xc2, xc3 = f32(0.1) * 1.0e6, 1.0 * 1.0e6, 1.0 * 1.0e6
    dz, dxx, dyy = 0.05e6, 0.5e6, 0.5e6
    AA, B, s_period = 10.0, f32(0.05), 240.0
    tdep = math.sin(qt * 2.0 * pi / s_period)
    X = [_view(P, P.x[..., d]) for d in range(3)]
    rb = _view(P, w0[..., v["rhob"]])
    for idx in np.ndindex(*P.nx):
        xx, yy, zz = X[1][idx] - xc2, X[2][idx] - xc3, X[0][idx] - xc1
        exp_z = math.exp(-(zz * zz) / (dz * dz))
        exp_x = math.exp(-(xx * xx) / (dxx * dxx))
        exp_y = math.exp(-(yy * yy) / (dyy * dyy))
        exp_xyz = exp_x * exp_y * exp_z
        theta, phi = math.atan2(yy, xx), math.atan2(1.0, B)
        ux, uy = math.cos(theta + phi), math.sin(theta + phi)
        vvx = (ux / math.sqrt(ux * ux + uy * uy)) * exp_xyz * tdep * AA
        vvy = (uy / math.sqrt(ux * ux + uy * uy)) * exp_xyz * tdep * AA
        r = new[idx + (v["rho"],)] + rb[idx]
        new[idx + (v["m0"] + 2,)] = new[idx + (v["m0"] + 2,)] + r * vvx * qdt
        new[idx + (v["m0"] + 3,)] = new[idx + (v["m0"] + 3,)] + r * vvy * qdt
        new[idx + (v["e"],)] = new[idx + (v["e"],)] + r * (vvx * vvx + vvy * vvy + 0.0 * 0.0) * qdt / 2.0
    nadv = 2 * P.ndir + 2
    np.testing.assert_array_equal(got[..., :nadv], new[..., :nadv])
