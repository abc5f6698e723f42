"""Snapshot and parameter formats (CPU).

Golden inputs: tests/golden/*.ini were written by the reference's own
inipar/*.py scripts (see tests/golden/make_golden.py)."""
import os
import struct

import numpy as np
import pytest

from sac_b200 import fileio, params, problems

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_golden_briowu_ini_reads():
    s = fileio.read_ini(os.path.join(GOLD, "briowu-test12_np01_000.ini"))
    assert fileio.detect_type(os.path.join(GOLD, "briowu-test12_np01_000.ini")) == "ascii"
    assert (s.it, s.t, s.ndim, s.neqpar, s.nw) == (0, 0.0, 1, 3, 10)
    assert s.nx == (800,)
    np.testing.assert_array_equal(s.eqpar, [2.0, 0.0, 1.0])
    assert s.varnames.split()[:11] == ["x", "rhop", "m1", "m2", "Ep", "b1p", "b2p", "rhob", "Eb", "b1b", "b2b"]
    assert s.w[:400, 0].tolist() == [1.0] * 400 and s.w[400:, 0].tolist() == [0.125] * 400


def test_briowu_builder_matches_reference_initial_data():
    """problems.brio_wu reproduces inipar/briowu-test12.py on the mesh."""
    s = fileio.read_ini(os.path.join(GOLD, "briowu-test12_np01_000.ini"))
    P = problems.brio_wu(nx=800)
    mesh = P.w[2:-2]
    np.testing.assert_array_equal(mesh, s.w)
    np.testing.assert_allclose(P.x[2:-2, 0], s.x[:, 0], rtol=0, atol=1e-15)


@pytest.mark.parametrize("name,nw,gamma", [("riemann-test11_np01_000.ini", 7, 1.4),
                                           ("strongshock-test11_np01_000.ini", 7, None)])
def test_golden_other_shocktubes(name, nw, gamma):
    s = fileio.read_ini(os.path.join(GOLD, name))
    assert s.nw == nw and s.ndim == 1
    if gamma is not None:
        assert s.eqpar[0] == gamma
    assert np.isfinite(s.w).all()


def _snap(nx=(5, 4), nw=10, seed=0):
    rng = np.random.default_rng(seed)
    nd = len(nx)
    x = np.asfortranarray(rng.standard_normal(nx + (nd,)))
    w = np.asfortranarray(rng.standard_normal(nx + (nw,)))
    w[0, 0, 1] = 3e-16  # below the ASCII zero threshold
    return fileio.Snapshot("test_mhd22", 7, 0.25, nd, 5, nw, nx, np.array([5 / 3, 0, -1, 0, 1.0]),
                           "x y rho m1 m2 e b1 b2 eb rhob bg1 bg2 gamma eta grav1 grav2 nu", x, w)


def test_binary_roundtrip_and_record_layout(tmp_path):
    s = _snap()
    p = tmp_path / "a.out"
    fileio.write_binary(p, [s, s])
    got = fileio.read_binary(p)
    assert len(got) == 2
    for g in got:
        np.testing.assert_array_equal(g.w, s.w)
        np.testing.assert_array_equal(g.x, s.x)
        assert (g.it, g.t, g.ndim, g.neqpar, g.nw, g.nx) == (s.it, s.t, s.ndim, s.neqpar, s.nw, s.nx)
    raw = p.read_bytes()
    # fileheadout record: CHARACTER*400 between two 4-byte length markers
    assert struct.unpack_from("<i", raw, 0)[0] == 400
    assert struct.unpack_from("<i", raw, 404)[0] == 400
    # it,t,ndim,neqpar,nw: 4+8+4+4+4 bytes
    assert struct.unpack_from("<i", raw, 408)[0] == 24
    # with a 400-character header the readfileini auto rule (marker 24 at byte 88)
    # does not recognise the file, as in the reference (typefileini must be set)
    assert fileio.detect_type(p) == "special"
    assert fileio.read_snapshots(p, "binary")[-1].it == 7


def test_ascii_roundtrip(tmp_path):
    s = _snap()
    p = tmp_path / "a.ini"
    fileio.write_ascii(p, s)
    assert fileio.detect_type(p) == "ascii"
    g = fileio.read_ini(p)
    ref = np.where(np.abs(s.w) > 5e-16, s.w, 0.0)
    np.testing.assert_allclose(g.w, ref, rtol=1e-10, atol=0)
    assert g.w[0, 0, 1] == 0.0
    lines = p.read_text().splitlines()
    assert lines[1] == "      7  2.50000E-01  2  5 10"
    assert lines[2] == "   5   4"


def test_fortran_edit_descriptors():
    assert fileio._fmt_1pe(2.0, 13, 5) == "  2.00000E+00"
    assert fileio._fmt_1pe(-0.000123456, 13, 5) == " -1.23456E-04"
    assert fileio._fmt_1pe(9.999996, 13, 5) == "  1.00000E+01"
    assert fileio.format_log_line(12, 0.5, 0.01, [1.0, -2.0]) == \
        "     12  5.00000E-01  1.00000E-02  1.00000E+00 -2.00000E+00"


PAR = """
 &testlist
    teststr=' '
 /
 &filelist
    filenameini='data/x_np01.ini'
    filename=   'data/x.log',
                'data/x.out'
    typefileout='binary'
 /
 &savelist
    itsave(1,2)=0
    ditsave=5,5
 /
 &stoplist
    tmax=0.15, itmax=1000
 /
 &methodlist
    wnames='rho m1 m2 e b1 b2 eb rhob bg1 bg2'
    typefull=6*'cd4',4*'nul'
    typeadvance='fourstep'
    dimsplit=F
    smallp= 0.6d0
 /
 &boundlist
    typeB= 10*'periodic'
           10*'cont'
           10*'fixed' ! a comment
           10*'cont'
 /
 &paramlist
    courantpar=0.8D0
 /
"""


def test_namelist_reader():
    pf = params.read_par(PAR)
    assert pf.get("stoplist", "tmax") == 0.15 and pf.get("stoplist", "itmax") == 1000
    assert pf.get("methodlist", "typefull") == ["cd4"] * 6 + ["nul"] * 4
    assert pf.get("methodlist", "typeadvance") == "fourstep"
    assert pf.get("methodlist", "dimsplit") is False
    assert pf.get("methodlist", "smallp") == 0.6
    assert pf.get("filelist", "filename") == ["data/x.log", "data/x.out"]
    assert pf.get("paramlist", "courantpar") == 0.8
    assert pf.get("savelist", "ditsave") == [5, 5]
    types = params.typeB_from_par(pf, nw=10, nB=4)
    assert types[0] == ["periodic"] * 10 and types[2] == ["fixed"] * 10 and types[3] == ["cont"] * 10


def test_params_struct_layout():
    p = params.make_params(gamma=2.0, grav=[-1.0, 0, 0], typeadvance="fourstep", user=params.USR_STRAT,
                           userpar=[1.0, 2.0])
    assert p.gamma == 2.0 and p.grav[0] == -1.0 and p.typeadvance == b"fourstep"
    assert p.userpar[1] == 2.0 and p.user == params.USR_STRAT
    assert params.pack_typeB([["cont", "periodic"]]) == b"cont      periodic  "
