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


def _fill_regions(w, nd, lo, hi, idim, up, types, pair):
    """The first fill with user regions (src/vacgrid.t:227-471): region by region
    in order, each over its own limits (1-based lo/hi), reading the edge, inner
    edge, mirror or periodic pair outside it."""
    w = w.copy()
    for iB in range(len(types)):
        d = idim[iB] - 1
        box = tuple(slice(lo[iB][e] - 1, hi[iB][e]) for e in range(nd))
        a0, a1 = lo[iB][d] - 1, hi[iB][d] - 1

        def plane(i):
            return tuple(i if e == d else box[e] for e in range(nd))

        for iw in range(w.shape[-1]):
            t = types[iB][iw]
            a = w[..., iw]
            ixe = a0 - 1 if up[iB] else a1 + 1
            if t in ("cont", "fixed"):
                for i in range(a0, a1 + 1):
                    a[plane(i)] = a[plane(ixe)]
            elif t in ("cont1", "fixed1", "grad1"):
                ixf = ixe - 1 if up[iB] else ixe + 1
                for i in range(a0, a1 + 1):
                    n = abs(i - ixe)
                    a[plane(i)] = float(n + 1) * a[plane(ixe)] - float(n) * a[plane(ixf)]
            elif t == "periodic":
                j = pair[iB]
                src = tuple(slice(lo[j][e] - 1 + (2 if (e == d and up[iB]) else -2 if e == d else 0),
                                  hi[j][e] + (2 if (e == d and up[iB]) else -2 if e == d else 0))
                            for e in range(nd))
                a[box] = a[src]
            elif t in ("symm", "asymm"):
                m = 2 * a0 - 1 if up[iB] else 2 * a1 + 1
                for i in range(a0, a1 + 1):
                    a[plane(i)] = (-1.0 if t == "asymm" else 1.0) * a[plane(m - i)]
            else:
                raise ValueError(t)
    return w


def test_user_regions_first_fill():
    """Six regions in 2D: the defaults given explicitly (the x2 pair matched by
    direction, orientation and extent) plus a 'cont1' and a 'symm'/'asymm'
    sub-region of the lower x1 boundary that overwrite parts of the first region
    and of each other, in order."""
    P = problems.random_problem((10, 8), seed=31, types=["cont", "cont", "periodic", "periodic"])
    nw = 3 * P.ndir + 4
    G = [n + 4 for n in P.nx]
    lo = [[1, 1], [G[0] - 1, 1], [1, 1], [1, G[1] - 1], [1, 2], [1, 5]]
    hi = [[2, G[1]], [G[0], G[1]], [G[0], 2], [G[0], G[1]], [2, 6], [2, 9]]
    idim = [1, 1, 2, 2, 1, 1]
    up = [False, True, False, True, False, False]
    types = [["cont"] * nw, ["cont"] * nw, ["periodic"] * nw, ["periodic"] * nw, ["cont1"] * nw, ["symm"] * nw]
    types[5][1] = "asymm"
    from sac_b200 import params
    o = Oracle(P.params)
    o.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    o.set_boundaries(params.pack_typeB(types), len(types), regions=(lo, hi, idim, up))
    o.upload(P.w)
    o.getboundary(0.0)
    ref = _fill_regions(P.w, 2, lo, hi, idim, up, types, pair={2: 3, 3: 2})
    np.testing.assert_array_equal(o.download(), ref)


def test_explicit_default_regions_are_the_default_fill():
    P = problems.random_problem((9, 7, 6), seed=32, types=["cont1", "fixed", "periodic", "periodic", "symm", "cont"])
    G = [n + 4 for n in P.nx]
    lo, hi, idim, up = [], [], [], []
    for iB in range(6):
        d, u = iB // 2, iB % 2
        a, b = [1, 1, 1], list(G)
        if u:
            a[d] = G[d] - 1
        else:
            b[d] = 2
        lo.append(a), hi.append(b), idim.append(d + 1), up.append(bool(u))
    a = _util.start(Oracle, P)
    o = Oracle(P.params)
    o.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    o.set_boundaries(P.typeB_packed, P.nB, regions=(lo, hi, idim, up))
    o.upload(P.w)
    o.getboundary(0.0)
    np.testing.assert_array_equal(o.download(), a.download())
    _util.run(a, 2)
    _util.run(o, 2)
    np.testing.assert_array_equal(o.download(), a.download())


def _primitive(w, ndir, gamma):
    """src/vacphys0.t.mhd:31-52 on the whole grid: p (getpthermal) into e, v = m/rho_t into m."""
    w = w.copy()
    rho, rhob = w[..., 0], w[..., 3 * ndir + 4 - ndir - 1]
    rt = rho + rhob
    m = [w[..., 1 + C].copy() for C in range(ndir)]
    b = [w[..., ndir + 2 + C] for C in range(ndir)]
    bg = [w[..., 2 * ndir + 4 + C] for C in range(ndir)]
    m2 = sum_ordered([mc * mc for mc in m])
    q = 0.5 * m2 / rt
    q = q + 0.5 * sum_ordered([bc * bc for bc in b]) + sum_ordered([bc * gc for bc, gc in zip(b, bg)])
    w[..., ndir + 1] = (gamma - 1.0) * (w[..., ndir + 1] - q)
    for C in range(ndir):
        w[..., 1 + C] = m[C] / rt
    return w


def _conserve(w, ndir, gamma):
    """src/vacphys0.t.mhd:5-28: e from p, v and b; m = rho_t v."""
    w = w.copy()
    rt = w[..., 0] + w[..., 3 * ndir + 4 - ndir - 1]
    v = [w[..., 1 + C].copy() for C in range(ndir)]
    b = [w[..., ndir + 2 + C] for C in range(ndir)]
    bg = [w[..., 2 * ndir + 4 + C] for C in range(ndir)]
    w[..., ndir + 1] = (w[..., ndir + 1] / (gamma - 1.0) + 0.5 * (rt * sum_ordered([x * x for x in v])
                                                                  + sum_ordered([x * x for x in b]))
                        + sum_ordered([x * y for x, y in zip(b, bg)]))
    for C in range(ndir):
        w[..., 1 + C] = rt * v[C]
    return w


def sum_ordered(terms):
    s = terms[0].copy()
    for t in terms[1:]:
        s = s + t
    return s


def test_zero_boundary_first_fill():
    """'zero' on the lower x1 boundary of a 2D state (src/vacgrid.t:295-346): per
    variable in order, primitive over the whole grid, contCD4's copy of that
    variable, conserve; then the other regions."""
    P = problems.random_problem((10, 8), seed=33, types=["zero", "cont", "periodic", "periodic"])
    nd, ndir = P.ndim, P.ndir
    nw = 3 * ndir + 4
    gamma = P.params.gamma
    o = _util.start(Oracle, P)
    w = P.w.copy()
    lo = 2
    for iw in range(nw):
        w = _primitive(w, ndir, gamma)
        # the lower region is x1 = 0..1 (0-based): its plane ixmin copies ixmax+3,
        # its plane ixmax copies ixmax+2
        w[0, :, iw] = w[lo + 2, :, iw]
        w[1, :, iw] = w[lo + 1, :, iw]
        w = _conserve(w, ndir, gamma)
    ref = _fill_regions_default_rest(P, w)
    np.testing.assert_array_equal(o.download(), ref)


def _fill_regions_default_rest(P, w):
    """Regions 2..4 of the default set after a 'zero' region 1 (cont upper x1,
    periodic x2)."""
    w = w.copy()
    lo, hi = 2, 2 + P.nx[0] - 1
    for i in (hi + 1, hi + 2):
        w[i] = w[hi]
    n2 = P.nx[1]
    w[:, 0] = w[:, n2]
    w[:, 1] = w[:, n2 + 1]
    w[:, n2 + 2] = w[:, 2]
    w[:, n2 + 3] = w[:, 3]
    return w
