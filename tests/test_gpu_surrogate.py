"""The surrogate pipeline end to end at a small size (64 x 64 flux tubes): solver
trajectories from the batched FP32 solver, training with libsacfno.so's own
kernels, and the judged roll-out against the plain solver.

What the trained network gains over the method without it is measured by the
full-size run (python -m sac_b200.surrogate); here the test checks that training
works (the loss falls, the one-window prediction beats both the untrained
network and the no-change prediction) and that the judge accepts, rejects and
rolls back as specified."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from sac_b200 import build, problems, surrogate as sg  # noqa: E402

pytestmark = pytest.mark.gpu

N = (64, 64)
WIN, NWIN = 8, 8


@pytest.fixture(scope="module")
def trained():
    build.build()
    build.build_fno()
    omega_ac = problems.flux_tube(N).meta["omega_ac"]
    dt = sg.stable_dt(N, nsteps=24)
    ds = sg.Dataset(24, NWIN, S=N[1], F=N[0])
    A, om = sg.drivers(24, 5, omega_ac)
    sg.generate(ds, A, om, dt, WIN, n=N, log=lambda m: None)
    sx, sd = sg.channel_scales(ds, nsample=24)
    sur = sg.Surrogate(S=N[1], F=N[0], batch=8, seed=1, layers=2, hidden=64)
    sur.set_scales(sx, sd)
    pairs = np.array([(n, k) for n in range(20, 24) for k in range(NWIN)])
    before = sur.evaluate_loss(ds, pairs)
    hist, _ = sur.train(ds, epochs=40, lr=2e-3, log=lambda m: None)
    after = sur.evaluate_loss(ds, pairs)
    return dict(sur=sur, ds=ds, dt=dt, hist=hist, before=before, after=after, omega_ac=omega_ac)


def test_training_reduces_the_loss(trained):
    h = trained["hist"]
    assert h[-1][1] < 0.2 * h[0][1], h


def test_trained_network_beats_untrained_and_no_change(trained):
    b, a = trained["before"], trained["after"]
    # relative L2 of the predicted increment; predicting no change scores 1
    assert a["val_rel_l2_increment"] < 0.5, a
    assert a["val_rel_l2_increment"] < 0.5 * b["val_rel_l2_increment"], (b, a)


def test_judged_rollout_accepts_rejects_and_rolls_back(trained):
    sur, dt = trained["sur"], trained["dt"]
    A, om = sg.drivers(6, 77, trained["omega_ac"])
    strict = sg.rollout(sur, A, om, dt, WIN, NWIN, M=4, tol=0.0, n=N, log=lambda m: None)
    assert strict["judged"] == 2 * 6 and strict["rejected"] == strict["judged"]
    # every window rejected and rolled back: the result is the plain solver's,
    # with its own dt, at the same end time as the reference run
    assert strict["final_rel_l2_max"] < 1e-3, strict
    loose = sg.rollout(sur, A, om, dt, WIN, NWIN, M=4, tol=1e9, n=N, log=lambda m: None)
    assert loose["judged"] == 2 * 6
    free = sg.rollout(sur, A, om, dt, WIN, NWIN, M=10 ** 9, tol=1e-3, n=N, log=lambda m: None)
    assert free["judged"] == 0 and np.isfinite(free["final_rel_l2_max"])
