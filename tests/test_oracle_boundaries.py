"""The oracle's boundary fill against a numpy transcription of the Fortran (CPU).

getboundary (src/vacgrid.t:195-512) with the default regions of boundsetup
(src/vacgrid.t:9-160): region iB = 1..2*ndim in order, each the two ghost layers
along its dimension times the whole grid in the others, so that later regions
overwrite the corners that earlier ones wrote; within a region every variable in
order.  The first fill is compared, in which 'fixed', 'fixed1' and 'grad1' act as
'cont' and 'cont1' (their stored values are captured after it), with the types
mixed per variable and per region."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import problems

import _util


def _fill(P, w, fix=None):
    """getboundary on a copy of w (every variable, default regions).  fix: the
    values captured after the first fill (_capture); None for the first fill."""
    w = w.copy()
    nd = P.ndim
    for iB in range(2 * nd):
        d, up = iB // 2, iB % 2 == 1
        lo, hi = 2, 2 + P.nx[d] - 1  # mesh edges along d
        layers = (hi + 1, hi + 2) if up else (lo - 2, lo - 1)

        def at(i):
            return tuple(i if e == d else slice(None) for e in range(nd))

        for iw in range(w.shape[-1]):
            t = P.typeB[iB][iw]
            a = w[..., iw]
            if fix is not None and (iB, iw) in fix:
                e = hi if up else lo
                for n, i in enumerate(layers):
                    stored = fix[(iB, iw)][n]
                    a[at(i)] = stored + a[at(e)] if t == "grad1" else stored
                continue
            if t in ("cont", "fixed"):
                e = hi if up else lo
                for i in layers:
                    a[at(i)] = a[at(e)]
            elif t in ("cont1", "fixed1", "grad1"):
                e, f = (hi, hi - 1) if up else (lo, lo + 1)
                for i in layers:
                    n = abs(i - e)
                    a[at(i)] = float(n + 1) * a[at(e)] - float(n) * a[at(f)]
            elif t == "periodic":
                shift = -(hi - lo + 1) if up else (hi - lo + 1)
                for i in layers:
                    a[at(i)] = a[at(i + shift)]
            elif t in ("symm", "symm0", "asymm"):
                e = 2 * (hi + 1) - 1 if up else 2 * (lo - 1) + 1  # ixe = 2*ixmin-1 / 2*ixmax+1
                for i in layers:
                    a[at(i)] = a[at(e - i)]
                if t == "asymm":
                    for i in layers:
                        a[at(i)] = -a[at(i)]
            elif t == "contCD4":
                # upper: first layer from hi-1, second from hi-2; lower: the mirror
                src = {hi + 1: hi - 1, hi + 2: hi - 2} if up else {lo - 2: lo + 2, lo - 1: lo + 1}
                for i in layers:
                    a[at(i)] = a[at(src[i])]
            else:
                raise ValueError(t)
    return w


def _capture(P, w):
    """fixB after the first fill (src/vacgrid.t:476-507): the ghost values of
    'fixed' and 'fixed1' regions, and for 'grad1' their difference to the edge."""
    fix = {}
    nd = P.ndim
    for iB in range(2 * nd):
        d, up = iB // 2, iB % 2 == 1
        lo, hi = 2, 2 + P.nx[d] - 1
        layers = (hi + 1, hi + 2) if up else (lo - 2, lo - 1)
        e = hi if up else lo
        for iw in range(w.shape[-1]):
            t = P.typeB[iB][iw]
            if t in ("fixed", "fixed1", "grad1"):
                a = w[..., iw]
                at = lambda i: tuple(i if k == d else slice(None) for k in range(nd))  # noqa: E731
                fix[(iB, iw)] = [a[at(i)] - a[at(e)] if t == "grad1" else a[at(i)].copy() for i in layers]
    return fix


_KINDS = ["cont", "fixed", "cont1", "fixed1", "grad1", "symm", "symm0", "asymm", "contCD4"]


def _types(nd, nw, periodic_dims, seed):
    rng = np.random.default_rng(seed)
    out = []
    for iB in range(2 * nd):
        if iB // 2 in periodic_dims:
            out.append(["periodic"] * nw)
        else:
            out.append([_KINDS[k] for k in rng.integers(0, len(_KINDS), size=nw)])
    return out


@pytest.mark.parametrize("nx,periodic_dims,seed", [((12,), (), 1), ((12,), (0,), 2), ((10, 9), (), 3),
                                                   ((10, 9), (1,), 4), ((8, 7, 6), (), 5), ((8, 7, 6), (0, 2), 6)])
def test_first_fill_matches_numpy(nx, periodic_dims, seed):
    P = problems.random_problem(nx, ndir=3 if len(nx) > 1 else 2, seed=seed)
    nw = P.w.shape[-1]
    P.typeB = _types(len(nx), nw, periodic_dims, seed)
    # ghost values that differ from any extrapolation of the mesh, so that a
    # ghost cell the fill misses shows
    rng = np.random.default_rng(seed + 100)
    w0 = P.w.copy()
    ghost = np.ones(P.w.shape[:-1], dtype=bool)
    ghost[tuple(slice(2, 2 + n) for n in nx)] = False
    w0[ghost] = rng.standard_normal((int(ghost.sum()), nw))
    P.w = w0
    o = _util.start(Oracle, P)
    np.testing.assert_array_equal(o.download(), _fill(P, w0))


@pytest.mark.parametrize("nx,periodic_dims,seed", [((12,), (), 7), ((10, 9), (), 8), ((8, 7, 6), (1,), 9)])
def test_later_fill_restores_the_captured_values(nx, periodic_dims, seed):
    P = problems.random_problem(nx, ndir=3 if len(nx) > 1 else 2, seed=seed)
    nw = P.w.shape[-1]
    P.typeB = _types(len(nx), nw, periodic_dims, seed)
    o = _util.start(Oracle, P)
    first = o.download()
    fix = _capture(P, first)
    # a changed state, ghosts included, then the next fill
    rng = np.random.default_rng(seed + 200)
    w1 = first + 0.1 * rng.standard_normal(first.shape)
    o.upload(w1)
    o.getboundary(0.0)
    np.testing.assert_array_equal(o.download(), _fill(P, w1, fix))


def test_fills_match_for_random_shapes_and_types():
    """Hypothesis-drawn grids (1D-3D, 5 to 9 mesh cells per dimension), boundary
    types per region and variable and periodic dimensions: first and later fill."""
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @settings(max_examples=30, deadline=None, derandomize=True)
    @given(st.lists(st.integers(5, 9), min_size=1, max_size=3), st.integers(0, 7), st.integers(0, 2 ** 16))
    def check(nx, periodic_mask, seed):
        nd = len(nx)
        periodic_dims = tuple(d for d in range(nd) if (periodic_mask >> d) & 1)
        P = problems.random_problem(tuple(nx), ndir=3 if nd > 1 else 2, seed=seed)
        nw = P.w.shape[-1]
        P.typeB = _types(nd, nw, periodic_dims, seed)
        o = _util.start(Oracle, P)
        first = o.download()
        np.testing.assert_array_equal(first, _fill(P, P.w))
        w1 = first + 0.1 * np.random.default_rng(seed).standard_normal(first.shape)
        o.upload(w1)
        o.getboundary(0.0)
        np.testing.assert_array_equal(o.download(), _fill(P, w1, _capture(P, first)))
        o.close()

    check()
