"""A full RK4 step of the oracle against the numpy transcriptions composed (CPU).

advect's 'fourstep' (src/vac.t:439-455): w1 = w + dt/2 R(w), w2 = w + dt/2 R(w1),
w3 = w + dt R(w2), each advect1 (src/vac.t:490-549) adding centdiff4's flux
divergence and then addsource2's sources (gravity, hyperdiffusion) to its base,
and filling the boundaries (getboundary); then w1 = (w1 + 2 w2 + w3 - 4 w)/3 and
w = w + dt/6 R(w3) + w1 over the whole grid, ghosts and background included.
Composed from the transcriptions of test_oracle_centdiff, test_oracle_visc and
test_oracle_boundaries, it must equal the oracle's step bit for bit."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import params, problems

import _util
from test_oracle_boundaries import _capture, _fill
from test_oracle_centdiff import _getflux, _getptotal_bg, _gradient4, _mesh
from test_oracle_keeppositive import _keeppositive
from test_oracle_sources import _powell_step, _resist1_step, _resist_step
from test_oracle_visc import Visc


_MAXNU = [0.0]  # maxviscoef over the setnu calls since the last getdt
_FIX = [None]  # the fixB values captured after the first fill, when a test sets them


def _advect1(P, qdt, wct, base, floors=None, dims=None):
    """floors: (smallp, smallrho, vacuumrho) when smallfix is set, so that the fill
    starts with keeppositive on the mesh (src/vacgrid.t:220).  dims: the 0-based
    idimmin..idimmax of a dimensionally split sweep (default: all)."""
    v = problems.var_index(P.ndir)
    gamma = P.params.gamma
    dims = list(range(P.ndim)) if dims is None else dims
    new = _mesh(P, base).copy()
    # centdiff4 (src/vaccd.t:35-70): fluxes from wCT, background work from the output array
    for d in dims:
        vel = wct[..., v["m0"] + 1 + d] / (wct[..., v["rho"]] + wct[..., v["rhob"]])
        for iw in range(v["eb"]):
            f, transport = _getflux(wct, v, P.ndir, gamma, iw, d)
            if transport:
                f = f + vel * wct[..., iw]
            new[..., iw] = new[..., iw] - qdt * _gradient4(P, f, d)
            if iw == v["e"]:
                fb = _mesh(P, _getptotal_bg(base, v, P.ndir, gamma))
                new[..., iw] = new[..., iw] - qdt * _gradient4(P, vel, d) * fb
                for di in dims:
                    bgi = _mesh(P, base[..., v["bg0"] + 1 + di])
                    bgd = _mesh(P, base[..., v["bg0"] + 1 + d])
                    new[..., iw] = new[..., iw] + qdt * bgi * bgd * _gradient4(P, vel, di)
    # addsource2 -> specialsource with qdt*(idimmax-idimmin+1)/ndim (src/vaccd.t:73-75),
    # which rounds in 3D: gravity (src/vacusr.gravity.t:24-81), then hyperdiffusion
    qdt = qdt * (float(len(dims) - 1) + 1.0) / float(P.ndim)
    g = list(P.params.grav)
    rho = _mesh(P, wct[..., v["rho"]])
    rt = _mesh(P, wct[..., v["rho"]] + wct[..., v["rhob"]])
    # gravity acts along every dimension, whatever the sweep
    for d in range(P.ndim):
        if abs(g[d]) > 1e-99:
            new[..., v["m0"] + 1 + d] = new[..., v["m0"] + 1 + d] + qdt * g[d] * rho
    for d in range(P.ndim):
        if abs(g[d]) > 1e-99:
            new[..., v["e"]] = new[..., v["e"]] + qdt * g[d] * rho * _mesh(P, wct[..., v["m0"] + 1 + d]) / rt
    V = Visc(P, wct, qdt)
    new = V.step(new)
    _MAXNU[0] = max(_MAXNU[0], V.maxviscoef)
    # addsource (src/vacphys.mhd0.t:225-258): resistivity, then Powell's term
    if abs(P.params.eta) > 1e-99:
        new = (_resist1_step if P.params.compactres else _resist_step)(P, wct, qdt, P.params.eta, new)
    if P.params.divbfix and P.ndim > 1:
        new = _powell_step(P, wct, qdt, new)
    out = base.copy()
    out[tuple(slice(2, 2 + n) for n in P.nx)] = new
    if floors is not None:
        out[tuple(slice(2, 2 + n) for n in P.nx)] = _keeppositive(P, out, *floors)[0]
    return _fill(P, out, _FIX[0])


def _fourstep(P, w, dt, floors=None, dims=None):
    w1 = _advect1(P, dt / 2, w, w, floors, dims)
    w2 = _advect1(P, dt / 2, w1, w, floors, dims)
    w3 = _advect1(P, dt, w2, w, floors, dims)
    w1 = (w1 + 2.0 * w2 + w3 - 4.0 * w) / 3.0
    w = _advect1(P, dt / 6, w3, w, floors, dims)
    return w + w1


@pytest.mark.parametrize("nx,ndir,types", [
    ((24,), 2, ["cont", "symm"]),
    ((14, 12), 3, ["cont1", "contCD4", "periodic", "periodic"]),
    ((10, 9, 8), 3, ["periodic", "periodic", "cont", "asymm", "cont", "symm"]),
])
def test_rk4_step_matches_the_composed_transcriptions(nx, ndir, types):
    P = problems.random_problem(nx, ndir=ndir, seed=41, types=types, typeadvance="fourstep")
    o = _util.start(Oracle, P)
    w0 = o.download()
    dt = 0.2 * o.getdt(0)
    o.advect(dt, 0.0, 0)
    got = o.download()
    want = _fourstep(P, w0, dt)
    assert np.abs(got - w0).max() > 1e-6
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("nx,smallp,vac_frac", [((24,), 0.001, 0.1), ((12, 10), 0.001, 0.15),
                                                ((9, 8, 7), -1.0, 0.1)])
def test_rk4_step_with_keeppositive_matches_the_composed_transcriptions(nx, smallp, vac_frac):
    """smallfix: each of the four fills starts with keeppositive on the mesh of the
    array it fills, before the ghost layers and before the combinations read it."""
    ndir = 3 if len(nx) > 1 else 2
    types = ["cont", "symm", "periodic", "periodic", "cont", "cont"][: 2 * len(nx)]
    P = problems.random_problem(nx, ndir=ndir, seed=43, types=types, typeadvance="fourstep")
    v = problems.var_index(ndir)
    m = _util.mesh(P, P.w)
    floors = (smallp, float(np.quantile(m[..., v["rho"]] + m[..., v["rhob"]], vac_frac)), 0.9)
    P.params.smallfix = 1
    P.params.smallp, P.params.smallrho, P.params.vacuumrho = floors
    o = _util.start(Oracle, P)
    w0 = o.download()
    dt = 0.2 * o.getdt(0)
    o.advect(dt, 0.0, 0)
    got = o.download()
    want = _fourstep(P, w0, dt, floors)
    assert o.diag().nerror_toosmallp == 5
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("nx,compact", [((24,), 0), ((24,), 1), ((12, 10), 0), ((12, 10), 1), ((9, 8, 7), 1)])
def test_rk4_step_with_resistivity_and_powell_matches_the_composed_transcriptions(nx, compact):
    """Gravity, hyperdiffusion, then addsource's resistive term (either form) and
    Powell's, in every stage of a fourstep step."""
    ndir = 3 if len(nx) > 1 else 2
    types = ["cont", "symm", "periodic", "periodic", "cont1", "cont"][: 2 * len(nx)]
    P = problems.random_problem(nx, ndir=ndir, seed=44, types=types, typeadvance="fourstep")
    P.params.eta, P.params.compactres, P.params.divbfix = 0.02, compact, 1
    o = _util.start(Oracle, P)
    w0 = o.download()
    dt = 0.2 * o.getdt(0)
    o.advect(dt, 0.0, 0)
    got = o.download()
    np.testing.assert_array_equal(got, _fourstep(P, w0, dt))


@pytest.mark.parametrize("nx,types", [((24,), ["fixed", "grad1"]), ((12, 10), ["fixed1", "cont", "periodic", "periodic"]),
                                      ((9, 8, 7), ["periodic", "periodic", "grad1", "fixed", "fixed1", "symm"])])
def test_rk4_step_with_stored_boundaries_matches_the_composed_transcriptions(nx, types):
    """'fixed', 'fixed1' and 'grad1' regions: every fill of the step restores the
    values captured after the first fill (src/vacgrid.t:476-507)."""
    ndir = 3 if len(nx) > 1 else 2
    P = problems.random_problem(nx, ndir=ndir, seed=45, types=types, typeadvance="fourstep")
    o = _util.start(Oracle, P)
    w0 = o.download()
    dt = 0.2 * o.getdt(0)
    o.advect(dt, 0.0, 0)
    _FIX[0] = _capture(P, w0)
    try:
        want = _fourstep(P, w0, dt)
    finally:
        _FIX[0] = None
    np.testing.assert_array_equal(o.download(), want)


@pytest.mark.parametrize("nx,sweeps", [((12, 10), [[0], [1]]), ((12, 10), [[1], [0]]), ((9, 8, 7), [[0], [1], [2]]),
                                       ((9, 8, 7), [[2], [1], [0]])])
def test_split_sweeps_match_the_composed_transcriptions(nx, sweeps):
    """Dimensionally split sweeps (advance_expl, src/vac.t:310-325): one advect per
    dimension, its fluxes and background work along that dimension only and its
    sources scaled by 1/ndim, then the next sweep from the result."""
    P = problems.random_problem(nx, ndir=3, seed=46, types=["cont", "symm", "periodic", "periodic", "cont1",
                                                            "cont"][: 2 * len(nx)], typeadvance="fourstep")
    P.params.eta, P.params.divbfix = 0.02, 1
    o = _util.start(Oracle, P)
    w = o.download()
    dt = 0.2 * o.getdt(0)
    for dims in sweeps:
        o.advect(dt, 0.0, 0, idimmin=dims[0] + 1, idimmax=dims[0] + 1)
        w = _fourstep(P, w, dt, dims=dims)
    np.testing.assert_array_equal(o.download(), w)


def test_rk4_steps_for_random_shapes_and_options():
    """Hypothesis-drawn grids (1D-3D, 6 to 9 mesh cells per dimension), boundary
    types (the stored ones included), ndir, resistivity in either form and
    Powell's term: one fourstep step of the oracle, bit for bit."""
    from hypothesis import given, settings
    from hypothesis import strategies as st

    kinds = ["cont", "cont1", "symm", "asymm", "contCD4", "fixed", "fixed1", "grad1"]

    @settings(max_examples=12, deadline=None, derandomize=True)
    @given(st.lists(st.integers(6, 9), min_size=1, max_size=3), st.integers(0, 2 ** 16), st.booleans(),
           st.lists(st.sampled_from(kinds + ["periodic"]), min_size=3, max_size=3),
           st.sampled_from([0.0, 0.01]), st.booleans(), st.booleans())
    def check(nx, seed, ndir3, kind, eta, compact, divb):
        nd = len(nx)
        types = []
        for d in range(nd):
            types += ["periodic", "periodic"] if kind[d] == "periodic" else [kind[d], kinds[(seed + d) % len(kinds)]]
        P = problems.random_problem(tuple(nx), ndir=3 if (ndir3 or nd == 3) else max(nd, 2), seed=seed,
                                    types=types, typeadvance="fourstep")
        P.params.eta, P.params.compactres, P.params.divbfix = eta, int(compact), int(divb)
        o = _util.start(Oracle, P)
        w0 = o.download()
        dt = 0.2 * o.getdt(0)
        o.advect(dt, 0.0, 0)
        _FIX[0] = _capture(P, w0)
        try:
            want = _fourstep(P, w0, dt)
        finally:
            _FIX[0] = None
        np.testing.assert_array_equal(o.download(), want)
        o.close()

    check()


def _integrate(P, w, dt, method, pred):
    """advect's other time integrators (src/vac.t:402-476); w1 starts as a copy of w."""
    nul = lambda wct, base: _fill(P, base.copy())  # noqa: E731  advect1 with method 'nul'
    if method == "onestep":
        return _advect1(P, dt, w.copy(), w)
    if method == "twostep":
        w1 = _advect1(P, dt / 2, w, w) if pred == "cd4" else nul(w, w)
        return _advect1(P, dt, w1, w)
    if method == "threestep":
        w1 = _advect1(P, dt, w, w)
        w2 = 3 * 0.25 * w + 0.25 * w1
        w2 = _advect1(P, dt / 4, w1, w2)
        w = w / 3 + w2 * (2.0 / 3)
        return _advect1(P, dt * 2.0 / 3, w2, w)
    # sterck's first fraction is the single-precision literal 0.12 (src/vac.t:459)
    f = (dt * float(np.float32(0.12)), dt / 4, dt / 2) if method == "sterck" else (dt / 4, dt / 3, dt / 2)
    w1 = _advect1(P, f[0], w, w)
    w2 = _advect1(P, f[1], w1, w)
    w1 = _advect1(P, f[2], w2, w)
    return _advect1(P, dt, w1, w)


@pytest.mark.parametrize("method,pred", [("onestep", "nul"), ("twostep", "nul"), ("twostep", "cd4"),
                                          ("threestep", "nul"), ("sterck", "nul"), ("jameson", "nul")])
def test_other_integrators_match_the_composed_transcriptions(method, pred):
    P = problems.random_problem((14, 12), ndir=3, seed=42, types=["cont", "symm", "periodic", "periodic"],
                                typeadvance=method, courantpar=0.2)
    P.params.typepred = pred.encode()
    o = _util.start(Oracle, P)
    w0 = o.download()
    dt = o.getdt(0)
    o.advect(dt, 0.0, 0)
    np.testing.assert_array_equal(o.download(), _integrate(P, w0, dt, method, pred))


def test_second_dt_takes_the_viscous_limit_of_the_step():
    """getdt after an RK4 step: getdt_courant on the new state, getdt_visc with
    maxviscoef, the largest nu of every setnu call of the step, and dtdiffpar
    0.25 (src/vacusr.viscosity.t:509-542), and the saved dtgrav."""
    P = problems.random_problem((14, 12), ndir=3, seed=44, types=["cont", "symm", "periodic", "periodic"],
                                typeadvance="fourstep")
    o = _util.start(Oracle, P)
    w0 = o.download()
    dt0 = o.getdt(0)
    o.advect(0.5 * dt0, 0.0, 0)
    dt1 = o.getdt(1)
    _MAXNU[0] = 0.0
    w1 = _fourstep(P, w0, 0.5 * dt0)
    V = Visc(P, w1, 0.0)
    courantmax = max(float((_mesh(P, V.cmax(d)) / V.dx(0, d)).max()) for d in range(P.ndim))
    want = min(1.0e99, P.params.courantpar / courantmax)
    for d in range(P.ndim):
        dxm = V.dx(0, d)
        want = min(want, 0.25 / float(((_MAXNU[0] + 0.0) / (dxm * dxm)).max()))
    grav = list(P.params.grav)
    dtgrav = 1.0e99
    for d in range(P.ndim):
        m = max(float((abs(grav[d]) / V.dx(0, j)).max()) for j in range(P.ndim))
        dtgrav = min(dtgrav, 1.0 / np.sqrt(m))
    want = min(want, dtgrav)
    assert _MAXNU[0] > 0.0
    assert dt1 == want
