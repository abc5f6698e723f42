"""Parity of the batched path (sac_batch_* of libsacgpu.so) with the CPU oracle.

Every instance of a batch is an independent program-vac run: after n RK4 steps
with its own dt, each must match the oracle advancing that instance alone
(FP64: 1e-12 relative L2 per variable and the same time t; FP32: 1e-5)."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import batch, params, problems

import _util

pytestmark = pytest.mark.gpu

RTOL = 1e-12
FP32_RTOL = 1e-5


def _oracle_run(P, nsteps):
    o = _util.start(Oracle, P)
    dts = _util.run(o, nsteps)
    return o.download(), dts


def _batch_of(problems_, prm, group_cells=0):
    P0 = problems_[0]
    b = batch.Batch(prm, P0.ndim, P0.ndir, [P.nx for P in problems_], group_cells=group_cells)
    b.set_grid(np.concatenate([P.x.reshape(-1, order="F") for P in problems_]))
    b.set_boundaries(P0.typeB)
    b.upload(np.concatenate([P.w.reshape(-1, order="F") for P in problems_]))
    b.getboundary()
    return b


def _check(problems_, b, nsteps, rtol):
    b.advance(nsteps)
    t, dt, it = b.state()
    wall = b.download()
    for i, P in enumerate(problems_):
        wo, dts = _oracle_run(P, nsteps)
        wg = b.instance(wall, i)
        assert it[i] == nsteps
        err = _util.rel_l2(_util.mesh(P, wg), _util.mesh(P, wo))
        assert np.isfinite(wg).all()
        assert err.max() <= rtol, f"instance {i} {P.nx}: rel L2 per variable {err}"
        np.testing.assert_allclose(t[i], sum(dts), rtol=RTOL)
        np.testing.assert_allclose(dt[i], dts[-1], rtol=RTOL)
        # ghost layers too (the boundary fill is part of each stage)
        np.testing.assert_allclose(wg, wo, rtol=0, atol=max(1e-9, 1e3 * rtol) * np.abs(wo).max())


def _ot_problems(sizes, betas, precision=0):
    out = []
    for n, beta in zip(sizes, betas):
        P = problems.orszag_tang(n, beta=beta)
        P.params = batch.ot_params(precision=precision)
        out.append(P)
    return out


def test_ot_uneven_fp64():
    sizes = [(16, 24), (40, 16), (24, 24), (32, 48), (16, 16)]
    betas = [0.5, 2.0, 10.0, 1.3, 5.0]
    Ps = _ot_problems(sizes, betas)
    b = _batch_of(Ps, Ps[0].params)
    _check(Ps, b, 20, RTOL)


def test_ot_generator_matches_problems():
    gen = batch.OTBatch(4, nx=[(16, 24), (24, 16), (32, 32), (16, 40)], betas=[0.5, 1.0, 4.0, 9.5])
    Ps = _ot_problems(gen.nx, gen.beta)
    for i, P in enumerate(Ps):
        np.testing.assert_array_equal(gen.state(i), P.w)
        np.testing.assert_array_equal(gen.x(i), P.x)
    b = gen.make(Ps[0].params)
    _check(Ps, b, 10, RTOL)


def test_groups_split_the_intermediates():
    sizes = [(16, 24), (40, 16), (24, 24), (32, 48), (16, 16), (20, 28)]
    Ps = _ot_problems(sizes, [1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    b = _batch_of(Ps, Ps[0].params, group_cells=1500)  # several groups
    _check(Ps, b, 8, RTOL)


def test_gravity_viscosity_mixed_bounds_2d():
    types = ["cont", "cont1", "symm", "asymm"]
    Ps = [problems.random_problem(n, seed=s, types=types) for n, s in (((14, 12), 1), ((20, 10), 2), ((12, 18), 3))]
    prm = Ps[0].params
    for P in Ps:
        P.params = prm
    b = _batch_of(Ps, prm)
    _check(Ps, b, 12, RTOL)


def _divb_problems(dtpar=None):
    types = ["cont", "cont1", "periodic", "periodic"]
    Ps = [problems.random_problem(n, seed=s, types=types) for n, s in (((14, 12), 4), ((20, 10), 5))]
    prm = Ps[0].params
    prm.divbfix = 1
    if dtpar is not None:
        prm.dtpar = dtpar
    for P in Ps:
        P.params = prm
    return Ps, prm


def test_divbfix_2d_fp64():
    Ps, prm = _divb_problems()
    _check(Ps, _batch_of(Ps, prm), 12, RTOL)


def test_divbfix_2d_fp32():
    Ps, prm = _divb_problems(dtpar=2.0e-3)
    prm.precision = params.PREC_FP32
    b = _batch_of(Ps, prm)  # the batch keeps its own copy of the parameters
    prm.precision = params.PREC_FP64
    _check(Ps, b, 10, FP32_RTOL)


def _resistive_problems(ndim, dtpar=None, eta=0.01):
    if ndim == 2:
        types = ["cont", "cont1", "periodic", "periodic"]
        Ps = [problems.random_problem(n, ndir=3, seed=s, types=types) for n, s in (((14, 12), 6), ((20, 10), 7))]
    else:
        Ps = [problems.random_problem((n,), ndir=3, seed=n, types=["cont", "symm"]) for n in (40, 33)]
    prm = Ps[0].params
    prm.eta = eta
    prm.divbfix = 1 if ndim == 2 else 0
    if dtpar is not None:
        prm.dtpar = dtpar
    for P in Ps:
        P.params = prm
    return Ps, prm


@pytest.mark.parametrize("ndim,eta", [(1, 0.01), (2, 0.01), (2, 0.5)])
def test_resistive_fp64(ndim, eta):
    # at eta = 0.5 getdt_res sets dt, with dtdiffpar 0.5 at the first step and the
    # 0.25 that getdt_visc leaves after it
    Ps, prm = _resistive_problems(ndim, eta=eta)
    _check(Ps, _batch_of(Ps, prm), 12, RTOL)


def test_resistive_2d_fp32():
    Ps, prm = _resistive_problems(2, dtpar=2.0e-3)
    prm.precision = params.PREC_FP32
    b = _batch_of(Ps, prm)
    prm.precision = params.PREC_FP64
    _check(Ps, b, 10, FP32_RTOL)


def test_1d_instances():
    Ps = [problems.random_problem((n,), ndir=2, seed=n, types=["cont", "symm"]) for n in (40, 64, 33)]
    prm = Ps[0].params
    for P in Ps:
        P.params = prm
    b = _batch_of(Ps, prm)
    _check(Ps, b, 15, RTOL)


def test_tuned_tiles_give_the_same_result():
    sizes = [(48, 40), (64, 24), (24, 56)]
    Ps = _ot_problems(sizes, [0.7, 3.0, 8.0])
    b = _batch_of(Ps, Ps[0].params)
    tile, ms = b.tune()
    assert tile[0] * tile[1] <= 256 and ms > 0
    _check(Ps, b, 10, RTOL)


def test_advance_in_pieces_equals_one_call():
    sizes = [(16, 24), (24, 16)]
    Ps = _ot_problems(sizes, [1.0, 2.0])
    b1 = _batch_of(Ps, Ps[0].params)
    b2 = _batch_of(Ps, Ps[0].params)
    b1.advance(6)
    for _ in range(3):
        b2.advance(2)
    np.testing.assert_array_equal(b1.download(), b2.download())
    np.testing.assert_array_equal(b1.state()[0], b2.state()[0])


# The FP32 path computes its own dt from FP32 data; the hyperdiffusion
# coefficient behind the viscous limit is a ratio of differences that is set by
# rounding noise wherever a field is flat, so that dt can differ by percents
# from FP64's.  The FP32 tests therefore fix dt (dtpar) in both runs and measure
# the storage precision alone.
FP32_DT = 2.0e-3


def test_ot_uneven_fp32():
    sizes = [(16, 24), (40, 16), (24, 24)]
    betas = [0.5, 2.0, 10.0]
    Ps = _ot_problems(sizes, betas)
    for P in Ps:
        P.params.dtpar = FP32_DT
    prm32 = batch.ot_params(precision=params.PREC_FP32)
    prm32.dtpar = FP32_DT
    b = _batch_of(Ps, prm32)
    _check(Ps, b, 10, FP32_RTOL)


def test_unsupported_options_are_errors():
    from sac_b200 import abi
    prm = batch.ot_params()
    prm.typeadvance = b"twostep"
    with pytest.raises(abi.SacError):
        batch.Batch(prm, 2, 2, [(16, 16)])
    prm = batch.ot_params()
    prm.eta = -0.01  # a user specialeta
    with pytest.raises(abi.SacError):
        batch.Batch(prm, 2, 2, [(16, 16)])
    prm = batch.ot_params()
    b = batch.Batch(prm, 2, 2, [(16, 16)])
    P = problems.orszag_tang((16, 16))
    b.set_grid(P.x.reshape(-1, order="F"))
    with pytest.raises(abi.SacError):
        b.set_boundaries([["fixed"] * 10 for _ in range(4)])


def _tubes(sizes, amps, omegas, precision=0):
    out = []
    for n, a, om in zip(sizes, amps, omegas):
        P = problems.flux_tube(n, A=a, omega=om)
        P.params.precision = precision
        out.append(P)
    return out


def _tube_batch(Ps, prm):
    b = _batch_of(Ps, prm)
    b.set_driver([P.params.userpar[0] for P in Ps], [P.params.userpar[1] for P in Ps])
    return b


def test_flux_tube_drivers_per_instance_fp64():
    Ps = _tubes([(24, 20), (32, 16), (20, 28)], [1e-2, 3e-3, 1e-4], [0.7, 1.2, 2.3])
    b = _tube_batch(Ps, Ps[0].params)
    _check(Ps, b, 12, RTOL)


def test_flux_tube_drivers_per_instance_fp32():
    Ps = _tubes([(24, 20), (32, 16)], [1e-2, 1e-3], [0.9, 1.7])
    for P in Ps:
        P.params.dtpar = FP32_DT
    prm = problems.flux_tube((24, 20)).params
    prm.precision = params.PREC_FP32
    prm.dtpar = FP32_DT
    b = _tube_batch(Ps, prm)
    _check(Ps, b, 12, FP32_RTOL)


def test_flux_tube_zero_perturbation_is_stationary():
    Ps = _tubes([(24, 20), (16, 32)], [0.0, 0.0], [1.0, 1.0])
    b = _tube_batch(Ps, Ps[0].params)
    w0 = b.download()
    b.advance(5)
    np.testing.assert_array_equal(b.download(), w0)


def test_gather_scatter_round_trip():
    torch = pytest.importorskip("torch")
    Ps = _tubes([(24, 20), (32, 16)], [1e-2, 3e-3], [0.7, 1.2])
    b = _tube_batch(Ps, Ps[0].params)
    b.advance(3)
    buf = torch.empty(b.packed_size, dtype=torch.float64, device="cuda")
    b.gather(buf.data_ptr(), "f64")
    b.synchronize()
    wall = b.download()
    got = buf.cpu().numpy()
    off = 0
    for i, P in enumerate(Ps):
        m = _util.mesh(P, b.instance(wall, i))  # (nx1, nx2, nw)
        n = int(np.prod(P.nx))
        blk = got[off: off + 6 * n].reshape(6, P.nx[1], P.nx[0])  # variable, x2, x1 (x1 fastest)
        for iw in range(6):
            np.testing.assert_array_equal(blk[iw], m[..., iw].T)
        off += 6 * n
    buf.mul_(2.0)
    b.scatter(buf.data_ptr(), "f64")
    b.synchronize()
    wall2 = b.download()
    for i, P in enumerate(Ps):
        np.testing.assert_array_equal(_util.mesh(P, b.instance(wall2, i))[..., :6],
                                      2.0 * _util.mesh(P, b.instance(wall, i))[..., :6])


def test_tmaxexact_lands_every_instance_on_tmax():
    sizes = [(16, 24), (24, 16), (32, 32)]
    Ps = _ot_problems(sizes, [0.7, 3.0, 8.0])
    b = _batch_of(Ps, Ps[0].params)
    tmax = 0.03
    b.advance_to(tmax, chunk=4)
    t, dt, it = b.state()
    np.testing.assert_array_equal(t, np.full(3, tmax))
    wall = b.download()
    before = wall.copy()
    b.advance(3)  # finished instances stay untouched
    np.testing.assert_array_equal(b.download(), before)
    np.testing.assert_array_equal(b.state()[2], it)
    for i, P in enumerate(Ps):
        o = _util.start(Oracle, P)
        tt, k = 0.0, 0
        while tt < tmax:  # src/vac.t:82 tmaxexact
            d = min(o.getdt(k), tmax - tt + 1e-99)
            o.advect(d, tt, k)
            tt += d
            k += 1
        assert k == it[i]
        err = _util.rel_l2(_util.mesh(P, b.instance(wall, i)), _util.mesh(P, o.download()))
        assert err.max() <= RTOL, err
