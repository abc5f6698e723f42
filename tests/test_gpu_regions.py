"""User boundary regions (&boundlist ixB^LIM, idimB, upperB; boundsetup,
src/vacgrid.t:71-99) on the CUDA path against the CPU oracle.

With user regions getboundary fills the regions in order, later ones overwriting
earlier ones where they overlap (src/vacgrid.t:227-471): here the lower x1
boundary is split into a 'cont' part and a 'fixed' part that a later region
overwrites, and a periodic pair with shifted extents.  The FP64 bar is the
path's: the initial fill bit for bit, then 1e-12 relative L2 per variable."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import abi, params, problems

import _util

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _default_regions(P):
    """The 2*ndim default regions as explicit (1-based) limits."""
    nd = P.ndim
    G = [n + 4 for n in P.nx]
    lo, hi, idim, up = [], [], [], []
    for iB in range(2 * nd):
        d, u = iB // 2, iB % 2
        a = [1] * nd
        b = list(G)
        if u:
            a[d] = G[d] - 1
        else:
            b[d] = 2
        lo.append(a)
        hi.append(b)
        idim.append(d + 1)
        up.append(bool(u))
    return lo, hi, idim, up


def _split_problem(seed=21, nx=(16, 14), fixed_extra=True):
    """Default 2D regions with types cont/cont/periodic/periodic, plus two more
    regions on the lower x1 boundary: x2 rows 1..7 'fixed', then rows 5..10
    'cont1' (its overlap with the first wins)."""
    P = problems.random_problem(nx, seed=seed, types=["cont", "cont", "periodic", "periodic"])
    lo, hi, idim, up = _default_regions(P)
    nw = 3 * P.ndir + 4
    types = [list(t) for t in P.typeB]
    if fixed_extra:
        lo.append([1, 1]); hi.append([2, 7]); idim.append(1); up.append(False)
        types.append(["fixed"] * nw)
        lo.append([1, 5]); hi.append([2, 10]); idim.append(1); up.append(False)
        types.append(["cont1"] * nw)
    return P, params.pack_typeB(types), len(types), (lo, hi, idim, up)


def _start(cls, P, typeB, nB, regions):
    c = cls(P.params)
    c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    c.set_boundaries(typeB, nB, regions=regions)
    c.upload(P.w)
    c.getboundary(0.0)
    return c


def test_explicit_default_regions_equal_the_default_path():
    P = problems.random_problem((14, 12), seed=20, types=["cont", "fixed", "periodic", "periodic"])
    a = _util.start(abi.Context, P)
    b = _start(abi.Context, P, P.typeB_packed, P.nB, _default_regions(P))
    np.testing.assert_array_equal(a.download(), b.download())
    _util.run(a, 5)
    _util.run(b, 5)
    np.testing.assert_array_equal(a.download(), b.download())


@pytest.mark.parametrize("typeadvance", ["fourstep", "twostep", "onestep"])
def test_overlapping_user_regions(typeadvance):
    P, typeB, nB, regions = _split_problem()
    P.params.typeadvance = typeadvance.encode()
    o = _start(Oracle, P, typeB, nB, regions)
    g = _start(abi.Context, P, typeB, nB, regions)
    np.testing.assert_array_equal(g.download(), o.download())
    d_o = _util.run(o, 20)
    d_g = _util.run(g, 20)
    np.testing.assert_allclose(d_g, d_o, rtol=RTOL, atol=0)
    wo, wg = o.download(), g.download()
    err = _util.rel_l2(_util.mesh(P, wg), _util.mesh(P, wo))
    assert err.max() <= RTOL, err
    np.testing.assert_allclose(wg, wo, rtol=0, atol=1e-9 * np.abs(wo).max())


def test_user_regions_3d_fp32():
    """3D with a grad1 region on part of the upper x1 boundary, FP64 and FP32."""
    P = problems.random_problem((10, 8, 8), seed=22, types=["fixed", "cont", "periodic", "periodic", "cont", "symm"])
    lo, hi, idim, up = _default_regions(P)
    nw = 3 * P.ndir + 4
    lo.append([13, 1, 3]); hi.append([14, 6, 9]); idim.append(1); up.append(True)
    P.typeB = [list(t) for t in P.typeB] + [["grad1"] * nw]
    P.regions = (lo, hi, idim, up)
    o, g = _util.start(Oracle, P), _util.start(abi.Context, P)
    np.testing.assert_array_equal(g.download(), o.download())
    _util.run(o, 10)
    _util.run(g, 10)
    err = _util.rel_l2(_util.mesh(P, g.download()), _util.mesh(P, o.download()))
    assert err.max() <= RTOL, err
    e32, etw = _util.fp32_twin(P, 10)
    assert e32.max() <= 150.0 * etw.max(), (e32, etw)


def test_regions_outside_the_grid_or_into_the_mesh_are_refused():
    P, typeB, nB, (lo, hi, idim, up) = _split_problem()
    bad = ([list(x) for x in lo], [list(x) for x in hi], list(idim), list(up))
    bad[1][4] = [2, 99]  # beyond ixGhi2
    for cls in (Oracle, abi.Context):
        c = cls(P.params)
        c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
        with pytest.raises(abi.SacError) as e:
            c.set_boundaries(typeB, nB, regions=bad)
        assert e.value.status == 1  # SAC_ERR_ARG, boundsetup's die
    bad = ([list(x) for x in lo], [list(x) for x in hi], list(idim), list(up))
    bad[1][4] = [4, 7]  # reaches the mesh along x1
    c = abi.Context(P.params)
    c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    with pytest.raises(abi.SacError) as e:
        c.set_boundaries(typeB, nB, regions=bad)
    assert e.value.status == 5
