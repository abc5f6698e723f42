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
    # (src/vacio.t:357-359); compactres=T selects addsource_res1
    assert vac.Run(_par(tmp_path, "a"), context=Oracle).params.divbfix == 1
    assert vac.Run(_par(tmp_path, "b", method="divbfix=F"), context=Oracle).params.divbfix == 0
    with pytest.raises(ValueError):
        vac.Run(_par(tmp_path, "c", method="sourceunsplit=F"), context=Oracle)
    assert vac.Run(_par(tmp_path, "d", method="sourceunsplit=F divbfix=F"), context=Oracle).params.sourceunsplit == 0
    assert vac.Run(_par(tmp_path, "e", method="compactres=T"), context=Oracle).params.compactres == 1
    assert vac.Run(_par(tmp_path, "e2"), context=Oracle).params.compactres == 0
    with pytest.raises(NotImplementedError):
        vac.Run(_par(tmp_path, "f", method="divbconstrain=T"), context=Oracle)


def test_final_report_warns_of_a_dt_below_dtmin(tmp_path):
    """The loop stops at the first dt below dtmin and program vac warns of it
    after the loop (src/vac.t:117)."""
    par = _par(tmp_path, "m").replace("&stoplist itmax=20 /", "&stoplist itmax=20 dtmin=1.D0 /")
    r = vac.Run(par, context=Oracle).run(verbose=False)
    assert r.it == 0 and r.final_report() == [" Warning: dt<dtmin !!!"]


def test_smallfix_runs_keeppositive_and_reports(tmp_path):
    """smallfix=T with its floors from &methodlist: with the defaults (-1) the
    fills only count negative perturbed pressures and the snapshots equal those
    of a run without it; with floors the run changes, and the end report gives
    the first error and the count (src/vac.t:117-136, src/vacphys.t.mhd:36-40)."""
    ref = vac.Run(_par(tmp_path, "r"), context=Oracle).run(verbose=False)
    assert ref.final_report() == []
    cnt = vac.Run(_par(tmp_path, "c", method="smallfix=T"), context=Oracle).run(verbose=False)
    assert cnt.params.smallfix == 1 and cnt.params.smallp == -1.0
    for a, b in zip(_snapshots(tmp_path / "c.out"), _snapshots(tmp_path / "r.out")):
        np.testing.assert_array_equal(a.w, b.w)
    rep = cnt.final_report()
    assert rep[0].startswith("Too small pressure (code= 1) at it=") and rep[-1].endswith("Pressure below psmall")
    n = int(rep[2].split("occurred")[1].split("times")[0])
    assert 0 < n <= 1 + 4 * 20
    flo = vac.Run(_par(tmp_path, "f", method="smallfix=T smallp=0.2D0 smallrho=0.2D0 vacuumrho=0.15D0"),
                  context=Oracle).run(verbose=False)
    assert (flo.params.smallp, flo.params.smallrho, flo.params.vacuumrho) == (0.2, 0.2, 0.15)
    wf, wr = _snapshots(tmp_path / "f.out")[-1].w, _snapshots(tmp_path / "r.out")[-1].w
    assert np.isfinite(wf).all() and np.abs(wf - wr).max() > 1e-3
    assert "occurred    81 times" in flo.final_report()[2]


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


def test_2d_run_applies_the_default_powell_source(tmp_path):
    """A 2D par without divbfix runs with the Powell source (par/DEFAULT:46), in
    program vac's dimensionally split loop (xyyx): equal to the oracle driven by
    hand with divbfix=1 the same way, and different from divbfix=0."""
    from sac_b200 import params, problems

    P = problems.random_problem((14, 12), ndir=3, seed=45, types=["cont", "cont", "periodic", "periodic"],
                                grav=(-0.7, 0.3, 0.0), nu=1.0, courantpar=0.4)
    names = "x y rho m1 m2 m3 e b1 b2 b3 eb rhob bg1 bg2 bg3 gamma eta grav1 grav2 nu"
    eqpar = np.array([P.params.gamma, 0.0, -0.7, 0.3, 1.0])
    mesh = (slice(2, 16), slice(2, 14))
    snap = fileio.Snapshot("2D random state", 0, 0.0, 2, 5, 13, (14, 12), eqpar, names,
                           np.asfortranarray(P.x[mesh]), np.asfortranarray(P.w[mesh]))
    ini = tmp_path / "r2d.ini"
    fileio.write_binary(str(ini), [snap])
    par = f"""
 &filelist filenameini='{ini}' typefileini='binary'
    filename='{tmp_path}/r.log', '{tmp_path}/r.out' typefileout='binary' /
 &savelist ditsave=100,6 /
 &stoplist itmax=6 /
 &methodlist typefull=8*'cd4',5*'nul' typeadvance='fourstep' /
 &boundlist typeB=13*'cont',13*'cont',13*'periodic',13*'periodic' /
 &paramlist courantpar=0.4 /
"""
    r = vac.Run(par, user="gravvisc", context=Oracle)
    assert r.params.divbfix == 1 and r.dimsplit
    r.run(verbose=False)
    got = fileio.read_binary(str(tmp_path / "r.out"))[-1]
    assert got.it == 6

    def by_hand(divbfix):
        prm = r.params
        prm.divbfix = divbfix
        o = Oracle(prm)
        o.set_grid(2, 3, r.ixGhi, r.ixM, r.x)
        o.set_boundaries(params.pack_typeB(r.types), 4)
        o.upload(r.w)
        o.getboundary(0.0)
        t = 0.0
        for it in range(6):
            dt = o.getdt(it)
            order = (1, 2) if it % 2 == 0 else (2, 1)  # typedimsplit 'xyyx'
            for d in order:
                o.advect(dt, t, it, method="cd4", iws=r.iws, idimmin=d, idimmax=d)
            t += dt
        w = o.download()
        o.close()
        return w[mesh]

    np.testing.assert_array_equal(got.w, by_hand(1))
    assert np.abs(got.w - by_hand(0)).max() > 1e-10


def _par_io(tmp, tag, extra_file="", itmax=5):
    return f"""
 &filelist filenameini='{INI}'
    filename='{tmp}/{tag}.log', '{tmp}/{tag}.out'
    typefileout='binary' {extra_file} /
 &savelist itsave(1,2)=0 ditsave=100,1 /
 &stoplist itmax={itmax} /
 &methodlist wnames='rhop m1 m2 Ep b1p b2p rhob Eb b1b b2b'
    typefull=6*'cd4',4*'nul' typeadvance='fourstep' /
 &boundlist typeB=40*'cont' /
 &paramlist courantpar=0.8 /
"""


def test_snapshotout_starts_a_new_file_every_n_saves(tmp_path):
    # savefile (src/vacio.t:901-958): after every snapshotout saves the output
    # continues in filename_<number of the next save>
    vac.Run(_par_io(tmp_path, "s", "snapshotout=2"), user="gravvisc", context=Oracle).run(verbose=False)
    its = {name: [s.it for s in _snapshots(tmp_path / name)] for name in ("s.out", "s.out_3", "s.out_5")}
    assert its == {"s.out": [0, 1], "s.out_3": [2, 3], "s.out_5": [4, 5]}


def test_fullgridout_saves_the_ghost_cells(tmp_path):
    r = vac.Run(_par_io(tmp_path, "f", "fullgridout=T", itmax=2), user="gravvisc", context=Oracle)
    r.run(verbose=False)
    last = _snapshots(tmp_path / "f.out")[-1]
    assert last.it == 2 and last.nx == tuple(r.ixGhi)
    np.testing.assert_array_equal(last.w, r.ctx.download())


def test_log_lines_hold_the_volume_weighted_means(tmp_path):
    """savefilelog_default (src/vacio.t:1094-1149): it, t, dt and, per variable,
    sum(dvolume w)/volume over the mesh, written (i7,100(1pe13.5))."""
    import _util

    r = vac.Run(_par(tmp_path, "m"), user="gravvisc", context=Oracle).run(verbose=False)
    snaps = {s.it: s for s in _snapshots(tmp_path / "m.out")}
    lines = open(tmp_path / "m.log").read().splitlines()[2:]
    dv = _util.gridsetup1_dx(r)[2:-2, 0]  # 1D: dvolume = dx on the mesh
    # the log saves every 5 steps from it=5; the .out file also at it=0 (itsave(1,2)=0)
    assert [int(x[:7]) for x in lines] == [5, 10, 15, 20]
    for line in lines:
        it = int(line[:7])
        vals = [float(line[7 + 13 * k: 20 + 13 * k]) for k in range((len(line) - 7) // 13)]
        s = snaps[it]
        assert vals[0] == pytest.approx(s.t, rel=1e-5, abs=1e-12)
        want = (dv[:, None] * s.w).sum(axis=0) / dv.sum()
        np.testing.assert_allclose(vals[2:2 + r.nw], want, rtol=1e-5, atol=1e-9)


def test_residual_stops_a_converged_run_and_is_logged(tmp_path):
    """residmin: program vac stops once ||w_n+1 - w_n|| (src/vac.t:88-98) falls
    below it, and the log gains a residual column."""
    base = _par(tmp_path, "c", itmax=200).replace("&stoplist itmax=200 /", "&stoplist itmax=200 residmin=3.D-3 /")
    r = vac.Run(base, user="gravvisc", context=Oracle)
    assert r.use_residual
    r.run(verbose=False)
    assert r.it < 200 and r.residual < 3e-3
    # the residual the driver used is that of the last step, recomputed here
    lines = open(tmp_path / "c.log").read().splitlines()
    assert lines[1].rstrip().endswith("residual")
    last = lines[-1]
    assert float(last[-13:]) == pytest.approx(r.residual, rel=1e-5)


def test_cputimemax_stops_the_run(tmp_path):
    base = _par(tmp_path, "p", itmax=100000).replace("&stoplist itmax=100000 /", "&stoplist itmax=100000 cputimemax=0.D0 /")
    r = vac.Run(base, user="gravvisc", context=Oracle).run(verbose=False)
    assert r.it == 0  # the time budget is spent before the first step


def test_par_eqpar_and_fileheadout_override_the_initial_file(tmp_path):
    base = _par(tmp_path, "q", itmax=2).replace("typefull=6*'cd4',4*'nul'",
                                                "typefull=6*'cd4',4*'nul' eqpar(1)=1.4D0 fileheadout='par header'")
    r = vac.Run(base, user="gravvisc", context=Oracle)
    assert r.params.gamma == 1.4 and r.eqpar[0] == 1.4
    r.run(verbose=False)
    snap = _snapshots(tmp_path / "q.out")[-1]
    # setheaderstrings: the physics suffix and the gravity module's parameter names
    assert snap.header.strip() == "par header_mhd12" and snap.eqpar[0] == 1.4
    assert snap.varnames.split()[-1] == "grav1" and "gamma eta" in snap.varnames


def test_slowsteps_scale_the_first_steps(tmp_path):
    """slowsteps=3 (src/vac.t:79): dt times 1-(1-k/3)^2 for the steps k=1, 2."""
    from sac_b200 import params

    base = _par(tmp_path, "w", itmax=4).replace("&paramlist courantpar=0.8 /", "&paramlist courantpar=0.8 slowsteps=3 /")
    r = vac.Run(base, user="gravvisc", context=Oracle)
    r.run(verbose=False)
    got = _snapshots(tmp_path / "w.out")[-1]

    o = Oracle(r.params)
    o.set_grid(1, 2, r.ixGhi, r.ixM, r.x)
    o.set_boundaries(params.pack_typeB(r.types), 2)
    o.upload(r.w)
    o.getboundary(0.0)
    t = 0.0
    for it in range(4):
        dt = o.getdt(it)
        if 3 > it + 1:
            q = 1.0 - (it + 1.0) / 3
            dt = dt * (1.0 - q * q)
        o.advect(dt, t, it, method="cd4", iws=r.iws)
        t += dt
    w = o.download()
    o.close()
    assert got.t == t
    np.testing.assert_array_equal(got.w, w[2:-2])
