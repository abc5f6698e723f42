"""sac_getdt_static, the getdt whose reduction scratch is a file-scope device
array (it allocates nothing), against sac_getdt.

Two contexts hold the same state: one takes its dt from sac_getdt, the other
from sac_getdt_static, and each advances with its own dt.  Two calls in a row
must give bit-identical dt, and the states stay identical after each step.
This file is collected last so that the test also runs after every other GPU
test in the same process (the scratch address is looked up once per device)."""
import ctypes

import numpy as np
import pytest

from sac_b200 import abi, params, problems

import _util

pytestmark = pytest.mark.gpu

MAX_CELLS = 33554432  # SAC_STATIC_MAX_CELLS


def _getdt_static(c, it):
    fn = c.lib.sac_getdt_static
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    fn.restype = ctypes.c_int
    dt = ctypes.c_double(0.0)
    st = fn(c.h, ctypes.byref(dt), int(it))
    if st != 0:
        raise abi.SacError(st, (c.lib.sac_last_error(c.h) or b"").decode())
    return dt.value


def _cases():
    strat = problems.stratified(n=(16, 12, 12))
    rnd3 = problems.random_problem((12, 10, 8), seed=5, types=["cont", "fixed", "periodic", "periodic",
                                                              "symm", "cont1"])
    rnd2 = problems.random_problem((24, 18), seed=6, types=["periodic", "periodic", "cont", "asymm"])
    f32 = problems.random_problem((20, 14), seed=7)
    f32.params.precision = params.PREC_FP32
    return [strat, rnd3, rnd2, f32]


@pytest.mark.parametrize("k", range(4))
def test_two_calls_in_a_row_match_getdt(k):
    P = _cases()[k]
    a = _util.start(abi.Context, P)
    b = _util.start(abi.Context, P)
    t = 0.0
    for it in range(2):
        da = a.getdt(it)
        db = _getdt_static(b, it)
        assert da == db, (it, da, db)
        a.advect(da, t, it)
        b.advect(db, t, it)
        t += da
        np.testing.assert_array_equal(a.download(), b.download())


def test_mesh_beyond_the_static_scratch_is_refused():
    n = MAX_CELLS + 1
    x = problems.make_grid((n,), (0.0,), (1.0,))
    w = problems.empty_state((n,), 2)
    v = problems.var_index(2)
    w[:, v["rho"]] = 1.0
    w[:, v["e"]] = 1.0
    prm = params.make_params(gamma=5.0 / 3.0, courantpar=0.4, typeadvance="fourstep",
                             user=params.USR_NONE)
    P = problems.Problem("uniform1d", 1, 2, (n,), prm, x, w, problems.uniform_types(1, v["nw"], "cont"))
    c = _util.start(abi.Context, P)
    del w, x
    with pytest.raises(abi.SacError) as e:
        _getdt_static(c, 0)
    assert e.value.status == 5 and str(MAX_CELLS) in str(e.value)
    assert c.getdt(0) > 0.0  # sac_getdt still covers it
    c.close()
