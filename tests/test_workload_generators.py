"""The seeded generators of the batched and surrogate workloads, on the CPU: the
uneven Orszag-Tang batch (sizes, betas, states against problems.orszag_tang) and
the flux tube's drivers and their features.  The GPU runs reproduce only if
these are deterministic and draw from the stated ranges."""
import math

import numpy as np

from sac_b200 import batch, problems, surrogate


def test_ot_sizes_and_betas_are_seeded_and_in_range():
    s1, s2 = batch.ot_sizes(512, seed=0), batch.ot_sizes(512, seed=0)
    assert s1 == s2 and batch.ot_sizes(512, seed=1) != s1
    allowed = set(batch.OT_SIZES)
    assert all(nx in allowed and ny in allowed for nx, ny in s1)
    assert set(batch.OT_SIZES) == set(range(64, 513, 32))
    nx = np.array([a for a, _ in s1])
    ny = np.array([b for _, b in s1])
    assert abs(np.corrcoef(nx, ny)[0, 1]) < 0.2  # drawn independently
    b1 = batch.ot_betas(4096, seed=0)
    np.testing.assert_array_equal(b1, batch.ot_betas(4096, seed=0))
    assert b1.min() >= 0.5 and b1.max() <= 10.0 and abs(b1.mean() - 5.25) < 0.2


def test_ot_generator_states_equal_the_problem_states():
    gen = batch.OTBatch(3, nx=[(16, 24), (24, 16), (32, 32)], betas=[0.5, 4.0, 9.5])
    for i, (n, beta) in enumerate(zip(gen.nx, gen.beta)):
        P = problems.orszag_tang(n, beta=beta)
        np.testing.assert_array_equal(gen.state(i), P.w)
        np.testing.assert_array_equal(gen.x(i), P.x)
    w = gen.w_concat()
    assert w.size == sum(gen.state(i).size for i in range(3))


def test_ot_thermal_pressure_gives_the_instance_beta():
    gen = batch.OTBatch(2, nx=[(32, 32), (32, 32)], betas=[0.7, 6.0])
    P = problems.orszag_tang((32, 32), beta=0.7)
    v = problems.var_index(2)
    for i, beta in enumerate(gen.beta):
        w = gen.state(i)
        # m_l and b_l sit at m0 + l and b0 + l (l = 1, 2); the background is zero
        rho = w[..., v["rho"]]
        m = w[..., v["m0"] + 1:v["m0"] + 3]
        b = w[..., v["b0"] + 1:v["b0"] + 3]
        kin = 0.5 * (m ** 2).sum(-1) / rho
        mag = 0.5 * (b ** 2).sum(-1)
        p = (gen.gamma - 1) * (w[..., v["e"]] - kin - mag)
        np.testing.assert_allclose(p, beta * gen.B0 ** 2 / 2.0, rtol=1e-12)
    assert P.ndim == 2


def test_surrogate_drivers_and_features():
    om_ac = problems.flux_tube((64, 64)).meta["omega_ac"]
    A, om = surrogate.drivers(2000, 0, om_ac)
    A2, om2 = surrogate.drivers(2000, 0, om_ac)
    np.testing.assert_array_equal(A, A2)
    np.testing.assert_array_equal(om, om2)
    assert A.min() >= 1e-4 and A.max() <= 1e-2  # log-uniform in [1e-4, 1e-2]
    assert abs(np.log10(A).mean() + 3.0) < 0.05
    assert om.min() >= 0.5 * om_ac and om.max() <= 2.0 * om_ac
    t = 0.123
    f = surrogate.features_host(A[:5], om[:5], np.full(5, t), om_ac)
    assert f.shape == (5, surrogate.NFEAT) and f.dtype == np.float32
    np.testing.assert_allclose(f[:, 0], np.sin(om[:5] * t), rtol=1e-6)
    np.testing.assert_allclose(f[:, 1], np.cos(om[:5] * t), rtol=1e-6)
    np.testing.assert_allclose(f[:, 3], np.log10(A[:5]) + 3.0, rtol=1e-6)
    assert math.isfinite(float(f.sum()))
