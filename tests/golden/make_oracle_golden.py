"""Regenerate the oracle's golden outputs in tests/golden (oracle_*.out).

Each case runs the CPU oracle through program vac's loop (getdt, then advect)
for a fixed number of steps from a seeded initial state and writes the full
grid, ghosts included, in VAC's binary .out format.  tests/test_oracle_golden.py
re-runs the cases and requires the oracle to reproduce these files bit for bit,
so that any change of the oracle's arithmetic shows.  Run from the repository
root:  python tests/golden/make_oracle_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from sac_b200 import fileio, problems  # noqa: E402


def cases():
    """name -> (Problem, steps)."""
    bw = problems.brio_wu(nx=128)
    r2 = problems.random_problem((16, 12), ndir=3, seed=46, types=["cont", "fixed", "periodic", "periodic"])
    r2.params.divbfix = 1
    r2.params.eta = 0.01
    st = problems.stratified(n=(12, 10, 10), amp=0.05)
    return {"oracle_briowu128_050": (bw, 50), "oracle_random2d_divb_eta_030": (r2, 30),
            "oracle_stratified12_020": (st, 20)}


def option_cases():
    """name -> (Problem, steps) for the options off by default: the Orszag-Tang
    vortex with keeppositive's floors (smallfix) and the compact resistive source
    (compactres)."""
    ot = problems.orszag_tang((32, 32))
    ot.params.smallfix = 1
    ot.params.smallp, ot.params.smallrho, ot.params.vacuumrho = 0.5, 2.75, 2.75
    ot.params.eta, ot.params.compactres = 0.01, 1
    return {"oracle_ot32_smallfix_compactres_020": (ot, 20)}


def run(P, steps, ctx_cls=None):
    """The case through program vac's loop on ctx_cls (default: the oracle);
    returns the full grid and the final time."""
    import _util

    if ctx_cls is None:
        from oracle.oracle import Oracle as ctx_cls
    o = _util.start(ctx_cls, P)
    t = 0.0
    for it in range(steps):
        dt = o.getdt(it)
        o.advect(dt, t, it)
        t += dt
    w = o.download()
    o.close()
    return w, t


def snapshot(P, w, t, steps):
    names = " ".join(["x%d" % (d + 1) for d in range(P.ndim)] + ["w%d" % (i + 1) for i in range(w.shape[-1])])
    return fileio.Snapshot("oracle golden", steps, t, P.ndim, 1, w.shape[-1], tuple(w.shape[:-1]),
                           np.array([P.params.gamma]), names, np.asfortranarray(P.x), np.asfortranarray(w))


def main():
    for name, (P, steps) in {**cases(), **option_cases()}.items():
        w, t = run(P, steps)
        fileio.write_binary(os.path.join(HERE, name + ".out"), [snapshot(P, w, t, steps)])
        print("wrote", name + ".out")


if __name__ == "__main__":
    main()
