"""The fused 2D stage of the batched path (one kernel per tile computing the
fluxes, setnu's quotients and the update in shared memory) against the
three-pass stage and the CPU oracle.

FP64: the fused stage computes every value with the same device functions in the
same order as the three passes, so the states agree bit for bit, and each
instance matches the oracle advancing it alone to 1e-12 relative L2.  Tiles of
both shapes (32x8, 16x8) cover instances whose sizes are not multiples of the
tile, so partial tiles and instance edges are exercised.  FP32: each path is
compiled with contraction, so the two FP32 forms are held to the oracle's FP32
tolerance on a fixed dt."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import abi, batch, params, problems

import _util
from test_gpu_batch import FP32_DT, FP32_RTOL, _batch_of, _ot_problems, _tube_batch, _tubes

pytestmark = pytest.mark.gpu

RTOL = 1e-12
SIZES = [(40, 24), (64, 72), (24, 56), (96, 33), (70, 64)]
BETAS = [0.6, 2.5, 9.0, 1.3, 4.0]


def _pair(Ps, prm, shape):
    a = _batch_of(Ps, prm)
    a.set_stage(False)
    f = _batch_of(Ps, prm)
    f.set_stage(True, shape)
    return a, f


@pytest.mark.parametrize("shape", [0, 1])
def test_fused_equals_three_passes_fp64(shape):
    Ps = _ot_problems(SIZES, BETAS)
    a, f = _pair(Ps, Ps[0].params, shape)
    a.advance(8)
    f.advance(8)
    np.testing.assert_array_equal(f.download(), a.download())
    ta, dta, ita = a.state()
    tf, dtf, itf = f.state()
    np.testing.assert_array_equal(tf, ta)
    np.testing.assert_array_equal(dtf, dta)


def test_fused_matches_the_oracle_fp64():
    Ps = _ot_problems(SIZES[:3], BETAS[:3])
    f = _batch_of(Ps, Ps[0].params)
    f.set_stage(True, 0)
    nsteps = 10
    f.advance(nsteps)
    t, dt, it = f.state()
    wall = f.download()
    for i, P in enumerate(Ps):
        o = _util.start(Oracle, P)
        dts = _util.run(o, nsteps)
        err = _util.rel_l2(_util.mesh(P, f.instance(wall, i)), _util.mesh(P, o.download()))
        assert err.max() <= RTOL, (i, err)
        np.testing.assert_allclose(t[i], sum(dts), rtol=RTOL)


def test_fused_flux_tubes_with_drivers_fp64():
    Ps = _tubes([(24, 20), (40, 16), (20, 36)], [1e-2, 3e-3, 1e-4], [0.7, 1.2, 2.3])
    a = _tube_batch(Ps, Ps[0].params)
    a.set_stage(False)
    f = _tube_batch(Ps, Ps[0].params)
    f.set_stage(True, 1)
    a.advance(10)
    f.advance(10)
    np.testing.assert_array_equal(f.download(), a.download())


def test_fused_fp32_against_the_oracle():
    """FP32 storage on a fixed dt: the sizes and bar of the batch's FP32 test."""
    sizes = [(16, 24), (40, 16), (24, 24)]
    Ps = _ot_problems(sizes, [0.5, 2.0, 10.0])
    for P in Ps:
        P.params.dtpar = FP32_DT
    prm32 = batch.ot_params(precision=params.PREC_FP32)
    prm32.dtpar = FP32_DT
    f = _batch_of(Ps, prm32)
    f.set_stage(True, 0)
    f.advance(10)
    wall = f.download()
    for i, P in enumerate(Ps):
        o = _util.start(Oracle, P)
        _util.run(o, 10)
        err = _util.rel_l2(_util.mesh(P, f.instance(wall, i)), _util.mesh(P, o.download()))
        assert err.max() <= FP32_RTOL, (i, err)


def test_fused_fp32_close_to_three_passes():
    """The two FP32 forms round differently (each compiled with contraction): on
    a fixed dt they stay within the FP32 bar of each other at the larger sizes."""
    Ps = _ot_problems(SIZES, BETAS)
    prm32 = batch.ot_params(precision=params.PREC_FP32)
    prm32.dtpar = FP32_DT
    a, f = _pair(Ps, prm32, 0)
    a.advance(5)
    f.advance(5)
    wa, wf = a.download(), f.download()
    for i, P in enumerate(Ps):
        err = _util.rel_l2(_util.mesh(P, f.instance(wf, i)), _util.mesh(P, a.instance(wa, i)))
        assert err.max() <= FP32_RTOL, (i, err)


def test_tuner_reports_both_forms():
    Ps = _ot_problems(SIZES, BETAS)
    b = _batch_of(Ps, Ps[0].params)
    b.tune()
    fused, shape, ms3, msf = b.stage()
    assert ms3 > 0 and msf > 0 and shape in (0, 1)
    assert fused == (msf < ms3)
    c = _batch_of(Ps, Ps[0].params)
    c.set_stage(False)
    b.advance(4)
    c.advance(4)
    np.testing.assert_array_equal(b.download(), c.download())


def test_fused_refused_where_it_does_not_apply():
    prm = batch.ot_params()
    prm.divbfix = 1
    Ps = _ot_problems([(16, 16)], [1.0])
    b = _batch_of(Ps, prm)
    with pytest.raises(abi.SacError) as e:
        b.set_stage(True, 0)
    assert e.value.status == 5
    P1 = [problems.random_problem((40,), ndir=2, seed=3, types=["cont", "symm"])]
    b1 = _batch_of(P1, P1[0].params)
    with pytest.raises(abi.SacError):
        b1.set_stage(True, 0)
