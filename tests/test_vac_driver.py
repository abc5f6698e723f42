"""program vac on top of the C-ABI (sac_b200.vac): parameter file, initial
snapshot, save schedule, .out snapshots and .log lines in the reference's
formats.  The CPU test drives it through the oracle; the GPU test runs the same
parameter file on the device and compares the files it writes with the
oracle's."""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from sac_b200 import fileio, vac

HERE = os.path.dirname(os.path.abspath(__file__))
INI = os.path.join(HERE, "golden", "briowu-test12_np01_000.ini")


def _par(tmp, tag, itmax=20, method=""):
    return f"""
 &filelist filenameini='{INI}'
    filename='{tmp}/{tag}.log', '{tmp}/{tag}.out'
    typefileout='binary' /
 &savelist itsave(1,2)=0 ditsave=5,5 /
 &stoplist itmax={itmax} /
 &methodlist wnames='rhop m1 m2 Ep b1p b2p rhob Eb b1b b2b'
    typefull=6*'cd4',4*'nul' typeadvance='fourstep' {method} /
 &boundlist typeB=40*'cont' /
 &paramlist courantpar=0.8 /
"""


def _snapshots(path):
    return fileio.read_binary(str(path))


def test_driver_on_the_oracle_writes_the_schedule(tmp_path):
    r = vac.Run(_par(tmp_path, "o"), user="gravvisc", context=Oracle).run(verbose=False)
    assert r.it == 20
    snaps = _snapshots(tmp_path / "o.out")
    assert [s.it for s in snaps] == [0, 5, 10, 15, 20]
    log = open(tmp_path / "o.log").read().splitlines()
    assert len(log) >= 5 and np.isfinite(snaps[-1].w).all()


def test_source_switches_follow_the_par(tmp_path):
    # divbfix defaults to T (par/DEFAULT:46) and needs unsplit sources
    # (src/vacio.t:357-359); compactres=T selects addsource_res1, not built
    assert vac.Run(_par(tmp_path, "a"), context=Oracle).params.divbfix == 1
    assert vac.Run(_par(tmp_path, "b", method="divbfix=F"), context=Oracle).params.divbfix == 0
    with pytest.raises(ValueError):
        vac.Run(_par(tmp_path, "c", method="sourceunsplit=F"), context=Oracle)
    assert vac.Run(_par(tmp_path, "d", method="sourceunsplit=F divbfix=F"), context=Oracle).params.sourceunsplit == 0
    with pytest.raises(NotImplementedError):
        vac.Run(_par(tmp_path, "e", method="compactres=T"), context=Oracle)


@pytest.mark.gpu
def test_driver_on_the_device_matches_the_oracle(tmp_path):
    vac.Run(_par(tmp_path, "o"), user="gravvisc", context=Oracle).run(verbose=False)
    vac.Run(_par(tmp_path, "g"), user="gravvisc").run(verbose=False)
    so, sg = _snapshots(tmp_path / "o.out"), _snapshots(tmp_path / "g.out")
    assert [s.it for s in sg] == [s.it for s in so]
    for a, b in zip(sg, so):
        assert a.t == pytest.approx(b.t, rel=1e-12)
        err = np.linalg.norm((a.w - b.w).ravel()) / np.linalg.norm(b.w.ravel())
        assert err <= 1e-12, (a.it, err)
    lo = open(tmp_path / "o.log").read().splitlines()
    lg = open(tmp_path / "g.log").read().splitlines()
    assert len(lo) == len(lg)
