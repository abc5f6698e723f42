"""The oracle reproduces its committed golden outputs bit for bit (CPU).

tests/golden/oracle_*.out were written by tests/golden/make_oracle_golden.py:
Brio-Wu (nx=128, 50 steps), a 2D random state with the Powell and resistive
sources and a fixed boundary (30 steps), and the 3D stratified atmosphere with
its driver (20 steps), and the Orszag-Tang vortex with keeppositive's floors and
the compact resistive source (20 steps), each through program vac's
getdt/advect loop, full grid with ghosts.  A change of the oracle's arithmetic
fails here."""
import os
import sys

import numpy as np
import pytest

from sac_b200 import fileio

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_oracle_golden as G  # noqa: E402


ALL = {**G.cases(), **G.option_cases()}


@pytest.mark.parametrize("name", sorted(ALL))
def test_oracle_reproduces_its_golden_output(name):
    P, steps = ALL[name]
    w, t = G.run(P, steps)
    ref = fileio.read_binary(os.path.join(HERE, "golden", name + ".out"))[-1]
    assert ref.it == steps and ref.t == t
    np.testing.assert_array_equal(w, ref.w)
