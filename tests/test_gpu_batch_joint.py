"""FP64 and FP32-perturbation instances advanced together (sac_batch_join), in
both join forms: joint kernels, where every kernel of the RK4 step walks the
tiles of an FP64 batch and of an FP32 batch in one persistent launch, and two
branches of one graph, each batch's own kernels.

- The FP64 instances advance bit for bit as the same batch advanced alone on the
  fused stage (the joint kernels run the FP64 tile bodies with the FP64 units'
  rounding rules), with their own t and dt; in the two-branch form the FP32
  instances do too.
- The FP32 instances, on a fixed dt, match the oracle advancing each alone within
  the batch's FP32 bar, and an FP32 batch advanced alone within the same bar (the
  joint unit computes FP32 without contraction, the FP32 unit with it).
- Flux tubes with per-instance drivers in both precisions.
- The join's refusals, the calls a joined batch refuses, and unjoining (also by
  destroying either batch)."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import abi, batch, params

import _util
from test_gpu_batch import FP32_DT, FP32_RTOL, _batch_of, _ot_problems, _tube_batch, _tubes

pytestmark = pytest.mark.gpu

RTOL = 1e-12
ERR_ARG, ERR_STATE, ERR_UNSUPPORTED = 1, 2, 5  # sac_status, include/sac_gpu.h
SIZES64 = [(40, 24), (64, 72), (24, 56)]
BETAS64 = [0.6, 2.5, 9.0]
SIZES32 = [(16, 24), (40, 16), (24, 24), (96, 33)]
BETAS32 = [0.5, 2.0, 10.0, 1.3]


def _pair(dtpar=None, shape=0):
    P64 = _ot_problems(SIZES64, BETAS64)
    P32 = _ot_problems(SIZES32, BETAS32)
    prm64 = batch.ot_params()
    prm32 = batch.ot_params(precision=params.PREC_FP32)
    if dtpar is not None:
        for P in P64 + P32:
            P.params.dtpar = dtpar
        prm64.dtpar = prm32.dtpar = dtpar
    b64 = _batch_of(P64, prm64)
    b64.set_stage(True, shape)
    b32 = _batch_of(P32, prm32)
    return P64, P32, prm64, prm32, b64, b32


@pytest.mark.parametrize("shape,form", [(0, 0), (1, 0), (0, 1)])
def test_fp64_instances_as_alone(shape, form):
    P64, P32, prm64, prm32, b64, b32 = _pair(shape=shape)
    alone = _batch_of(P64, prm64)
    alone.set_stage(True, shape)
    b64.join(b32)
    b64.set_join_form(form)
    b64.advance(8)
    alone.advance(8)
    np.testing.assert_array_equal(b64.download(), alone.download())
    t, dt, it = b64.state()
    ta, dta, ita = alone.state()
    np.testing.assert_array_equal(t, ta)
    np.testing.assert_array_equal(dt, dta)
    np.testing.assert_array_equal(it, ita)
    # the FP32 instances advanced too, with their own dt
    t32, dt32, it32 = b32.state()
    assert (it32 == 8).all() and (t32 > 0).all()
    assert np.isfinite(b32.download()).all()
    if form == 1:  # each batch's own kernels: the FP32 ones as an FP32 batch alone
        alone32 = _batch_of(P32, prm32)
        alone32.set_stage(True, shape)
        alone32.advance(8)
        np.testing.assert_array_equal(b32.download(), alone32.download())


def test_join_times_both_forms_and_keeps_the_faster():
    P64, P32, prm64, prm32, b64, b32 = _pair()
    assert b64.join_info()[0] == -1
    b64.join(b32)
    form, ms_joint, ms_forked = b64.join_info()
    assert ms_joint > 0 and ms_forked > 0
    assert form == (1 if ms_forked < ms_joint else 0)
    with pytest.raises(abi.SacError):
        b64.set_join_form(2)
    with pytest.raises(abi.SacError) as e:  # only the lead sets the form
        b32.set_join_form(0)
    assert e.value.status == ERR_STATE


def test_both_against_the_oracle_on_a_fixed_dt():
    P64, P32, prm64, prm32, b64, b32 = _pair(dtpar=FP32_DT)
    b64.join(b32)
    nsteps = 10
    b64.advance(nsteps)
    w64, w32 = b64.download(), b32.download()
    for i, P in enumerate(P64):
        o = _util.start(Oracle, P)
        _util.run(o, nsteps)
        err = _util.rel_l2(_util.mesh(P, b64.instance(w64, i)), _util.mesh(P, o.download()))
        assert err.max() <= RTOL, ("fp64", i, err)
    for i, P in enumerate(P32[:3]):
        o = _util.start(Oracle, P)
        _util.run(o, nsteps)
        err = _util.rel_l2(_util.mesh(P, b32.instance(w32, i)), _util.mesh(P, o.download()))
        assert err.max() <= FP32_RTOL, ("fp32", i, err)
    t, dt, it = b32.state()
    np.testing.assert_allclose(t, nsteps * FP32_DT, rtol=1e-12)


def test_fp32_instances_close_to_an_fp32_batch_alone():
    P64, P32, prm64, prm32, b64, b32 = _pair(dtpar=FP32_DT)
    alone = _batch_of(P32, prm32)
    alone.set_stage(True, 0)
    b64.join(b32)
    b64.advance(5)
    alone.advance(5)
    wj, wa = b32.download(), alone.download()
    for i, P in enumerate(P32):
        err = _util.rel_l2(_util.mesh(P, b32.instance(wj, i)), _util.mesh(P, alone.instance(wa, i)))
        assert err.max() <= FP32_RTOL, (i, err)


def test_flux_tubes_in_both_precisions():
    T64 = _tubes([(24, 20), (40, 16)], [1e-2, 3e-3], [0.7, 1.2])
    T32 = _tubes([(20, 36), (24, 20), (16, 32)], [1e-4, 1e-2, 2e-3], [2.3, 0.9, 1.5])
    for P in T64 + T32:
        P.params.dtpar = FP32_DT
    prm64 = type(T64[0].params).from_buffer_copy(T64[0].params)  # the drivers come per instance
    prm32 = type(prm64).from_buffer_copy(prm64)
    prm32.precision = params.PREC_FP32
    b64 = _tube_batch(T64, prm64)
    b32 = _tube_batch(T32, prm32)
    alone = _tube_batch(T64, prm64)
    for b in (b64, b32, alone):
        b.set_stage(True, 1)
    b64.join(b32)
    b64.advance(10)
    alone.advance(10)
    np.testing.assert_array_equal(b64.download(), alone.download())
    w32 = b32.download()
    for i, P in enumerate(T32):
        o = _util.start(Oracle, P)
        _util.run(o, 10)
        err = _util.rel_l2(_util.mesh(P, b32.instance(w32, i)), _util.mesh(P, o.download()))
        assert err.max() <= FP32_RTOL, (i, err)


def test_join_refusals():
    P64, P32, prm64, prm32, b64, b32 = _pair()
    with pytest.raises(abi.SacError) as e:  # the FP32 batch cannot lead
        b32.join(b64)
    assert e.value.status == ERR_ARG
    other64 = _batch_of(P64, prm64)
    with pytest.raises(abi.SacError):  # two FP64 batches
        b64.join(other64)
    prm_g = batch.ot_params(precision=params.PREC_FP32)
    prm_g.gamma = 1.4
    P_g = _ot_problems(SIZES32[:1], BETAS32[:1], precision=params.PREC_FP32)
    bg = _batch_of(P_g, prm_g)
    with pytest.raises(abi.SacError) as e:  # other parameters
        b64.join(bg)
    assert e.value.status == ERR_ARG
    prm_d = batch.ot_params()
    prm_d.divbfix = 1
    prm_d32 = batch.ot_params(precision=params.PREC_FP32)
    prm_d32.divbfix = 1
    bd64 = _batch_of(P64, prm_d)
    bd32 = _batch_of(P32, prm_d32)
    with pytest.raises(abi.SacError) as e:  # Powell's term keeps the three passes
        bd64.join(bd32)
    assert e.value.status == ERR_UNSUPPORTED


def test_joined_batches_refuse_what_would_break_the_join():
    P64, P32, prm64, prm32, b64, b32 = _pair()
    b64.join(b32)
    for call in (lambda: b32.advance(1), lambda: b32.tune(), lambda: b64.tune(),
                 lambda: b64.set_stage(False), lambda: b32.set_stage(True, 1)):
        with pytest.raises(abi.SacError) as e:
            call()
        assert e.value.status == ERR_STATE
    with pytest.raises(abi.SacError):
        b32.join(b64)
    with pytest.raises(abi.SacError):  # unjoin takes the lead
        b32.unjoin()


def test_unjoin_and_destroy_end_the_join():
    P64, P32, prm64, prm32, b64, b32 = _pair()
    alone64 = _batch_of(P64, prm64)
    alone64.set_stage(True, 0)
    b64.join(b32)
    b64.advance(2)
    alone64.advance(2)
    b64.unjoin()
    b32.advance(3)  # alone again, on its own stream
    b64.advance(1)
    alone64.advance(1)
    np.testing.assert_array_equal(b64.download(), alone64.download())
    t, dt, it = b32.state()
    assert (it == 5).all()
    # destroying the partner ends a join; the lead then advances alone
    b64.join(b32)
    b32.close()
    b64.advance(1)
    alone64.advance(1)
    np.testing.assert_array_equal(b64.download(), alone64.download())
