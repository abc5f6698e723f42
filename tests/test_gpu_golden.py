"""The CUDA path against the oracle's committed golden outputs (GPU).

The same cases as tests/test_oracle_golden.py (written by
tests/golden/make_oracle_golden.py), run through the C-ABI: the advanced
variables on the mesh within 1e-12 relative L2 per variable of the fixture and
the final time within 1e-12 relative.  The device keeps its background exact
where the reference's RK combinations let it drift by an ulp, so the
background and ghost cells are not compared."""
import os
import sys

import numpy as np
import pytest

from sac_b200 import abi, fileio

import _util

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_oracle_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(G.cases()))
def test_device_reproduces_the_golden_output(name, ctx_cls=None):
    P, steps = G.cases()[name]
    w, t = G.run(P, steps, ctx_cls or abi.Context)
    ref = fileio.read_binary(os.path.join(HERE, "golden", name + ".out"))[-1]
    assert ref.it == steps
    np.testing.assert_allclose(t, ref.t, rtol=1e-12, atol=0)
    nadv = 2 * P.ndir + 2
    err = _util.rel_l2(_util.mesh(P, w)[..., :nadv], _util.mesh(P, ref.w)[..., :nadv])
    assert np.isfinite(w).all()
    assert err.max() <= 1e-12, f"{name}: rel L2 per variable {err}"
