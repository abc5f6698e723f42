"""The compact resistive source (compactres=T, addsource_res1,
src/vacphys.mhdres.t:96-220) on the CUDA path against the CPU oracle: random
1D-3D states with a constant eta, with the Powell source, through the 'source'
method, and in FP32; the bars of the FP64 and FP32 paths (1e-12 and 1e-5
relative L2 per variable after the steps)."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import abi, batch, params, problems

import _util

pytestmark = pytest.mark.gpu

RTOL = 1e-12
FP32_RTOL = 1e-5


def _pair(P):
    return _util.start(Oracle, P), _util.start(abi.Context, P)


def _compare(P, o, g, rtol=RTOL):
    wo = _util.mesh(P, o.download())
    wg = _util.mesh(P, g.download())
    assert np.isfinite(wg).all()
    err = _util.rel_l2(wg, wo)[: 2 * P.ndir + 2]
    assert err.max() <= rtol, f"{P.name}: rel L2 per variable {err}"


def _steps(P, nsteps):
    o, g = _pair(P)
    d_o = _util.run(o, nsteps)
    d_g = _util.run(g, nsteps)
    np.testing.assert_allclose(d_g, d_o, rtol=1e-12, atol=0)
    _compare(P, o, g)


def _compact(P, eta):
    P.params.eta = eta
    P.params.compactres = 1
    return P


@pytest.mark.parametrize("nx,ndir", [((40,), 1), ((40,), 2), ((40,), 3), ((20, 16), 2), ((20, 16), 3),
                                     ((12, 10, 8), 3)])
def test_compact_resistive_random(nx, ndir):
    types = ["cont", "fixed", "periodic", "periodic", "cont", "symm"][: 2 * len(nx)]
    _steps(_compact(problems.random_problem(nx, ndir=ndir, seed=44, types=types), 0.01), 100)


def test_compact_resistive_dt_limit_binds():
    P = _compact(problems.random_problem((14, 12), ndir=3, seed=6, types=["cont", "cont1", "periodic", "periodic"]),
                 0.5)
    P.params.divbfix = 1
    _steps(P, 30)


def test_compact_resistive_with_divbfix_3d():
    P = _compact(problems.random_problem((12, 10, 8), seed=45,
                                         types=["cont", "cont", "periodic", "periodic", "fixed", "cont"]), 0.01)
    P.params.divbfix = 1
    _steps(P, 100)


def test_compact_resistive_source_method():
    P = _compact(problems.random_problem((16, 12), ndir=3, seed=46, types=["cont", "cont", "periodic", "periodic"]),
                 0.05)
    o, g = _pair(P)
    for k in range(3):
        o.advect(0.01, 0.01 * k, k, method="source")
        g.advect(0.01, 0.01 * k, k, method="source")
    _compare(P, o, g)


def test_fp32_compact_resistive_3d():
    P = _compact(problems.random_problem((12, 10, 8), seed=45,
                                         types=["cont", "cont", "periodic", "periodic", "fixed", "cont"]), 0.01)
    o = _util.start(Oracle, P)
    P.params.precision = params.PREC_FP32
    g = _util.start(abi.Context, P)
    dts = _util.run(o, 50)
    _util.run(g, 50, dts=dts)
    _compare(P, o, g, FP32_RTOL)


def test_batch_rejects_compactres():
    prm = batch.ot_params()
    prm.eta = 0.01
    prm.compactres = 1
    with pytest.raises(abi.SacError):
        batch.Batch(prm, 2, 2, [(16, 16)])
