"""The oracle's keeppositive against a numpy transcription of the Fortran (CPU).

keeppositive (src/vacphys.t.mhd:8-49), which getboundary runs on the mesh before the
ghost fill when smallfix is set (src/vacgrid.t:220): the vacuum state where
rho'+rhob < smallrho, the thermal pressure of getpthermal
(src/vacphys0.t.mhd:163-183) against max(0,smallp), the error count, and for
smallp > 0 the energy rebuilt from max(p,smallp) over the whole mesh, with the
kinetic term over the perturbed density alone as written there."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import problems

import _util


def _csum(terms):
    s = terms[0]
    for t in terms[1:]:
        s = s + t
    return s


def _keeppositive(P, w, smallp, smallrho, vacuumrho):
    """Mesh of w after keeppositive, whether the error fired, and minval(p)."""
    v = problems.var_index(P.ndir)
    g = P.params.gamma
    M = _util.mesh(P, w).copy()
    rho, e, eb, rhob = v["rho"], v["e"], v["eb"], v["rhob"]
    m = [v["m0"] + 1 + c for c in range(P.ndir)]
    b = [v["b0"] + 1 + c for c in range(P.ndir)]
    bg = [v["bg0"] + 1 + c for c in range(P.ndir)]
    vac = (M[..., rho] + M[..., rhob]) < smallrho
    for i in m:
        M[..., i][vac] = 0.0
    M[..., rho][vac] = (vacuumrho - M[..., rhob])[vac]
    b2 = _csum([M[..., i] * M[..., i] for i in b])
    M[..., e][vac] = (smallp / (g - 1.0) + 0.5 * b2 - M[..., eb])[vac]
    # getpthermal
    m2 = _csum([M[..., i] * M[..., i] for i in m])
    q = 0.5 * m2 / (M[..., rho] + M[..., rhob])
    q = q + 0.5 * b2 + _csum([M[..., i] * M[..., j] for i, j in zip(b, bg)])
    p = (g - 1.0) * (M[..., e] - q)
    low = bool((p < max(0.0, smallp)).any())
    if low and smallp > 0.0:
        M[..., e] = np.maximum(p, smallp) / (g - 1.0) + 0.5 * (m2 / M[..., rho] + b2) - M[..., eb]
    return M, low, p.min()


def _problem(nx, seed, smallp, vac_frac, vacuumrho=0.9):
    P = problems.random_problem(nx, ndir=3 if len(nx) > 1 else 2, seed=seed,
                                types=["periodic"] * (2 * len(nx)), typeadvance="onestep")
    v = problems.var_index(P.ndir)
    rt = _util.mesh(P, P.w)[..., v["rho"]] + _util.mesh(P, P.w)[..., v["rhob"]]
    smallrho = float(np.quantile(rt, vac_frac)) if vac_frac > 0 else -1.0
    P.params.smallfix = 1
    P.params.smallp = smallp
    P.params.smallrho = smallrho
    P.params.vacuumrho = vacuumrho
    return P, smallrho


@pytest.mark.parametrize("nx,smallp,vac_frac", [((24,), 0.02, 0.2), ((24,), -1.0, 0.0), ((12, 10), 0.02, 0.15),
                                                ((12, 10), 0.0, 0.3), ((8, 7, 6), 0.01, 0.1),
                                                ((8, 7, 6), -1.0, 0.25)])
def test_first_fill_matches_numpy(nx, smallp, vac_frac):
    P, smallrho = _problem(nx, 11 + len(nx), smallp, vac_frac)
    want, low, pmin = _keeppositive(P, P.w, smallp, smallrho, 0.9)
    o = _util.start(Oracle, P)
    got = _util.mesh(P, o.download())
    np.testing.assert_array_equal(got, want)
    if vac_frac > 0:  # the vacuum branch acted
        v = problems.var_index(P.ndir)
        assert (got[..., v["rho"]] + got[..., v["rhob"]] == 0.9).sum() > 0
    d = o.diag()
    # perturbed pressures of both signs: the error fires at every fill
    assert low and d.nerror_toosmallp == 1
    assert d.toosmallp_it == 0 and d.toosmallp_min == pmin
    o.close()


def test_errors_count_each_fill_and_keep_the_first_step():
    """nerror(toosmallp_) counts every fill that found a low pressure: four per
    'fourstep' step after the initial one; the first error's step stays."""
    P, smallrho = _problem((10, 9), 21, -1.0, 0.0)
    P.params.typeadvance = b"fourstep"
    o = _util.start(Oracle, P)
    assert o.diag().nerror_toosmallp == 1
    _util.run(o, 3, it0=7)
    d = o.diag()
    assert d.nerror_toosmallp == 1 + 3 * 4
    assert d.toosmallp_it == 0
    o.close()


def test_no_error_while_the_pressure_stays_above_the_floor():
    """smallp far below every perturbed pressure: neither count nor change."""
    P, _ = _problem((12, 10), 31, -1.0, 0.0)
    v = problems.var_index(P.ndir)
    P.w[..., v["e"]] += 5.0  # lifts p' well above 0 everywhere
    ref = _util.start(Oracle, P)
    P.params.smallfix = 0
    off = _util.start(Oracle, P)
    np.testing.assert_array_equal(ref.download(), off.download())
    assert ref.diag().nerror_toosmallp == 0
    ref.close()
    off.close()


def test_later_fill_matches_numpy():
    """A later fill on a changed mesh runs keeppositive again: the mesh equals
    the transcription applied to the uploaded state, and the count is 2."""
    P, smallrho = _problem((9, 8, 7), 41, 0.05, 0.0)
    v = problems.var_index(P.ndir)
    o = _util.start(Oracle, P)
    w1 = o.download()
    # a changed mesh energy, uploaded, then one more fill
    rng = np.random.default_rng(5)
    w2 = w1.copy()
    mesh = tuple(slice(2, 2 + n) for n in P.nx)
    w2[mesh + (v["e"],)] += 0.01 * rng.standard_normal(_util.mesh(P, w1)[..., 0].shape)
    o.upload(w2)
    o.getboundary(0.0)
    want, low, _ = _keeppositive(P, w2, 0.05, smallrho, 0.9)
    assert low
    np.testing.assert_array_equal(_util.mesh(P, o.download()), want)
    assert o.diag().nerror_toosmallp == 2
    o.close()


def test_first_fill_for_random_shapes_and_floors():
    """Hypothesis-drawn grids (1D-3D, 5 to 9 mesh cells per dimension), ndir and
    floors (smallp of either sign, smallrho from none to most cells): the first
    fill's mesh and error record equal the transcription's."""
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @settings(max_examples=25, deadline=None, derandomize=True)
    @given(st.lists(st.integers(5, 9), min_size=1, max_size=3), st.integers(0, 2 ** 16), st.booleans(),
           st.sampled_from([-1.0, 0.0, 0.003, 0.05]), st.sampled_from([0.0, 0.1, 0.6]))
    def check(nx, seed, ndir3, smallp, vac_frac):
        nd = len(nx)
        P = problems.random_problem(tuple(nx), ndir=3 if (ndir3 or nd == 3) else max(nd, 2), seed=seed,
                                    types=["periodic"] * (2 * nd), typeadvance="onestep")
        v = problems.var_index(P.ndir)
        rt = _util.mesh(P, P.w)[..., v["rho"]] + _util.mesh(P, P.w)[..., v["rhob"]]
        smallrho = float(np.quantile(rt, vac_frac)) if vac_frac > 0 else -1.0
        P.params.smallfix, P.params.smallp, P.params.smallrho, P.params.vacuumrho = 1, smallp, smallrho, 0.7
        want, low, pmin = _keeppositive(P, P.w, smallp, smallrho, 0.7)
        o = _util.start(Oracle, P)
        np.testing.assert_array_equal(_util.mesh(P, o.download()), want)
        d = o.diag()
        assert d.nerror_toosmallp == int(low)
        if low:
            assert d.toosmallp_min == pmin
        o.close()

    check()
