"""Parity of the CUDA path (libsacgpu.so through the C-ABI) with the CPU oracle.

The bar is the hot path's: FP64 results within 1e-12 relative L2 per variable of
the oracle after 100 steps (tolerance RTOL below), dt within 1e-12 relative.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import abi, params, problems

import _util

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _pair(P):
    o = _util.start(Oracle, P)
    g = _util.start(abi.Context, P)
    return o, g


def _compare(P, o, g, rtol=RTOL):
    wo = _util.mesh(P, o.download())
    wg = _util.mesh(P, g.download())
    err = _util.rel_l2(wg, wo)
    assert np.isfinite(wg).all()
    assert err.max() <= rtol, f"{P.name}: rel L2 per variable {err}"
    return err


def _steps(P, nsteps, **kw):
    o, g = _pair(P)
    d_o = _util.run(o, nsteps, **kw)
    d_g = _util.run(g, nsteps, **kw)
    np.testing.assert_allclose(d_g, d_o, rtol=1e-12, atol=0)
    return _compare(P, o, g)


def test_getboundary_initial_fill():
    P = problems.random_problem((14, 12), seed=11, types=["cont", "fixed", "periodic", "periodic"])
    o, g = _pair(P)
    np.testing.assert_array_equal(g.download(), o.download())


@pytest.mark.parametrize("types", [
    ["cont1", "grad1", "symm", "asymm"],
    ["fixed1", "contCD4", "symm0", "cont"],
    ["periodic", "periodic", "fixed", "cont1"],
])
def test_boundary_types_2d(types):
    P = problems.random_problem((12, 10), seed=12, types=types)
    o, g = _pair(P)
    np.testing.assert_array_equal(g.download(), o.download())
    _util.run(o, 5)
    _util.run(g, 5)
    _compare(P, o, g)


def test_briowu_100_steps():
    P = problems.brio_wu(nx=128)
    P.params.user = params.USR_GRAVVISC
    _steps(P, 100)


@pytest.mark.parametrize("ndir", [1, 2, 3])
def test_random_1d(ndir):
    P = problems.random_problem((40,), ndir=ndir, seed=3 + ndir)
    _steps(P, 100)


@pytest.mark.parametrize("ndir", [2, 3])
def test_random_2d(ndir):
    P = problems.random_problem((20, 16), ndir=ndir, seed=5, types=["cont", "fixed", "periodic", "periodic"])
    _steps(P, 100)


def test_random_3d_mixed_bounds():
    P = problems.random_problem((12, 10, 8), seed=6, types=["fixed", "cont", "periodic", "periodic", "cont", "symm"])
    _steps(P, 100)


def test_stratified_3d_driver():
    P = problems.stratified(n=(16, 12, 12), amp=0.05)
    _steps(P, 100)


def test_zero_perturbation_stays_zero():
    P = problems.stratified(n=(12, 10, 10), amp=0.0)
    g = _util.start(abi.Context, P)
    _util.run(g, 20)
    w = g.download()
    assert np.all(w[..., : 2 * P.ndir + 2] == 0.0)


@pytest.mark.parametrize("method,pred", [("onestep", "nul"), ("twostep", "nul"), ("twostep", "cd4"),
                                          ("threestep", "nul"), ("sterck", "nul"), ("jameson", "nul")])
def test_time_integrators(method, pred):
    P = problems.random_problem((16, 12), seed=7, types=["cont", "cont", "periodic", "periodic"],
                                typeadvance=method, courantpar=0.2)
    P.params.typepred = pred.encode()
    _steps(P, 20)


def test_dimensional_splitting():
    P = problems.random_problem((14, 12), seed=8, types=["cont", "cont", "periodic", "periodic"])
    _steps(P, 20, idim=[1, 2])


def test_slog_driver_with_alias():
    P = problems.random_problem((10, 8, 8), seed=9, user=params.USR_SLOG)
    # Slog lengths are in metres (Mm scale), x1 vertical
    P.x[...] *= 1.0e6
    P.params.alias_nu_grav3 = 1
    _steps(P, 10)


def test_source_method_only():
    P = problems.random_problem((16, 12), seed=10, types=["cont", "cont", "periodic", "periodic"])
    o, g = _pair(P)
    for k in range(5):
        dt = 0.01
        o.advect(dt, 0.01 * k, k, method="source")
        g.advect(dt, 0.01 * k, k, method="source")
    _compare(P, o, g)


# Powell's div B source (divbfix), src/vacphys.mhd0.t:263-297
@pytest.mark.parametrize("ndir", [2, 3])
def test_divbfix_random_2d(ndir):
    P = problems.random_problem((20, 16), ndir=ndir, seed=41, types=["cont", "fixed", "periodic", "periodic"])
    P.params.divbfix = 1
    _steps(P, 100)


def test_divbfix_random_3d():
    P = problems.random_problem((12, 10, 8), seed=42, types=["fixed", "cont", "periodic", "periodic", "cont", "symm"])
    P.params.divbfix = 1
    _steps(P, 100)


def test_divbfix_stratified_driver():
    P = problems.stratified(n=(16, 12, 12), amp=0.05)
    P.params.divbfix = 1
    _steps(P, 50)


def test_divbfix_source_method_and_splitting():
    P = problems.random_problem((16, 12), seed=43, types=["cont", "cont", "periodic", "periodic"])
    P.params.divbfix = 1
    o, g = _pair(P)
    for k in range(3):
        o.advect(0.01, 0.01 * k, k, method="source")
        g.advect(0.01, 0.01 * k, k, method="source")
    _compare(P, o, g)
    _util.run(o, 10, t0=0.03, it0=3, idim=[1, 2])
    _util.run(g, 10, t0=0.03, it0=3, idim=[1, 2])
    _compare(P, o, g)


# constant resistivity (addsource_res2 and getdt_res, src/vacphys.mhdres.t)
@pytest.mark.parametrize("nx,ndir", [((40,), 2), ((40,), 3), ((20, 16), 2), ((20, 16), 3), ((12, 10, 8), 3)])
def test_resistive_random(nx, ndir):
    types = ["cont", "fixed", "periodic", "periodic", "cont", "symm"][: 2 * len(nx)]
    P = problems.random_problem(nx, ndir=ndir, seed=44, types=types)
    P.params.eta = 0.01
    _steps(P, 100)


def test_resistive_dt_limit_binds():
    # getdt_res sets dt: dtdiffpar 0.5 at the first step, 0.25 after getdt_visc
    P = problems.random_problem((14, 12), ndir=3, seed=6, types=["cont", "cont1", "periodic", "periodic"])
    P.params.eta = 0.5
    P.params.divbfix = 1
    _steps(P, 30)


def test_resistive_with_divbfix_3d():
    P = problems.random_problem((12, 10, 8), seed=45, types=["cont", "cont", "periodic", "periodic", "fixed", "cont"])
    P.params.eta = 0.01
    P.params.divbfix = 1
    _steps(P, 100)


def test_resistive_source_method():
    P = problems.random_problem((16, 12), ndir=3, seed=46, types=["cont", "cont", "periodic", "periodic"])
    P.params.eta = 0.05
    o, g = _pair(P)
    for k in range(3):
        o.advect(0.01, 0.01 * k, k, method="source")
        g.advect(0.01, 0.01 * k, k, method="source")
    _compare(P, o, g)


def test_special_boundary_is_an_error():
    """'special' calls the user's specialbound, which the reference's user files
    define as die('not defined') (src/vacusr.f:1387-1399): an error here too."""
    P = problems.random_problem((12, 10), seed=48, types=["special", "cont", "periodic", "periodic"])
    g = abi.Context(P.params)
    g.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    with pytest.raises(abi.SacError):
        g.set_boundaries(P.typeB_packed, P.nB)


@pytest.mark.parametrize("where", ["lower", "upper", "both"])
def test_zero_boundary(where):
    """'zero' (src/vacgrid.t:295-346): the whole grid to primitive variables, the
    contCD4 copy, and back to conservative ones, once per variable that has it, so
    every fill re-rounds e and m everywhere; both paths do it in the same order."""
    types = {"lower": ["zero", "cont"], "upper": ["cont1", "zero"], "both": ["zero", "zero"]}[where]
    P = problems.random_problem((14, 12), seed=49, types=types + ["periodic", "periodic"])
    o, g = _pair(P)
    np.testing.assert_array_equal(g.download(), o.download())
    d_o = _util.run(o, 10)
    d_g = _util.run(g, 10)
    np.testing.assert_allclose(d_g, d_o, rtol=RTOL, atol=0)
    _compare(P, o, g)


def test_negative_eta_is_an_error():
    P = problems.random_problem((12, 10), seed=47, types=["cont", "cont", "periodic", "periodic"])
    P.params.eta = -0.01
    g = _util.start(abi.Context, P)
    with pytest.raises(abi.SacError):
        g.getdt(0)
    with pytest.raises(abi.SacError):
        g.advect(0.01, 0.0, 0)


def test_diag_matches_oracle():
    P = problems.random_problem((12, 10, 8), seed=6, types=["cont", "cont", "periodic", "periodic", "cont", "cont"])
    o, g = _pair(P)
    _util.run(o, 3)
    _util.run(g, 3)
    do, dg = o.diag(), g.diag()
    np.testing.assert_allclose(list(dg.wmean)[:P.nw], list(do.wmean)[:P.nw], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(dg.divb_l2, do.divb_l2, rtol=1e-10)
    np.testing.assert_allclose(dg.divb_linf, do.divb_linf, rtol=1e-10)


# ---------------------------------------------------------------------------
# FP32-perturbation path: advanced variables stored and updated in FP32,
# background, pressure/energy recovery and dt in FP64.  Tolerance: 1e-5
# relative L2 per variable against the FP64 oracle after 100 steps.
# ---------------------------------------------------------------------------
FP32_RTOL = 1e-5


def _fp32_steps(P, nsteps):
    o = _util.start(Oracle, P)
    P.params.precision = params.PREC_FP32
    g = _util.start(abi.Context, P)
    P.params.precision = params.PREC_FP64
    dts = _util.run(o, nsteps)
    _util.run(g, nsteps, dts=dts)
    wo = _util.mesh(P, o.download())
    wg = _util.mesh(P, g.download())
    err = _util.rel_l2(wg, wo)[: 2 * P.ndir + 2]
    assert np.isfinite(wg).all()
    assert err.max() <= FP32_RTOL, f"{P.name}: FP32 rel L2 per variable {err}"
    return err


def test_fp32_stratified_3d():
    _fp32_steps(problems.stratified(n=(16, 12, 12), amp=0.05), 100)


def test_fp32_random_2d():
    _fp32_steps(problems.random_problem((20, 16), seed=5, types=["cont", "fixed", "periodic", "periodic"]), 100)


def test_fp32_divbfix_2d():
    P = problems.random_problem((20, 16), seed=41, types=["cont", "fixed", "periodic", "periodic"])
    P.params.divbfix = 1
    _fp32_steps(P, 100)


def test_fp32_resistive_3d():
    P = problems.random_problem((12, 10, 8), seed=45, types=["cont", "cont", "periodic", "periodic", "fixed", "cont"])
    P.params.eta = 0.01
    P.params.divbfix = 1
    _fp32_steps(P, 100)


def test_fp32_zero_perturbation_stays_zero():
    P = problems.stratified(n=(12, 10, 10), amp=0.0)
    P.params.precision = params.PREC_FP32
    g = _util.start(abi.Context, P)
    _util.run(g, 20)
    assert np.all(g.download()[..., : 2 * P.ndir + 2] == 0.0)
