"""bench.py's choice of workload, on the CPU: the 512^3 line starts from the
precision-comparison configuration's 64 random modes and the 128^3 leg from
rest, the line's config says which, and the CPU sample is the same state on
the 128^3 cube."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402
from sac_b200 import problems  # noqa: E402


def test_initial_state_by_size():
    assert bench.perturb_for(512, "auto") == bench.MODES_AMP
    assert bench.perturb_for(128, "auto") is None
    assert bench.perturb_for(128, "modes") == bench.MODES_AMP
    assert bench.perturb_for(512, "rest") is None


def test_workload_states():
    rest = bench.workload(16, None)
    modes = bench.workload(16, bench.MODES_AMP)
    ref = problems.stratified(n=(16, 16, 16), perturb=bench.MODES_AMP)
    np.testing.assert_array_equal(modes.w, ref.w)  # seeded: the same state every run
    # the background is shared; the perturbation is zero at rest and of the stated amplitude with modes
    npv = 2 * rest.ndir + 2  # the advanced variables; the background follows them
    np.testing.assert_array_equal(rest.w[..., npv:], modes.w[..., npv:])
    assert np.abs(rest.w[..., 0]).max() == 0.0
    assert 0 < np.abs(modes.w[..., 0]).max() < 100 * bench.MODES_AMP


def test_config_names_the_state():
    assert "random modes" in bench.headline_config(512, 1, bench.MODES_AMP)["workload"]
    assert "at rest" in bench.headline_config(128, 1, None)["workload"]
    txt = bench.cpu_sample_text({"steps": 3, "seconds": 1.0, "n": 128, "threads": 4, "perturb": bench.MODES_AMP})
    assert "64 random modes" in txt and "128^3" in txt
