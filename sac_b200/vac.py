"""Host driver: the main program of the reference, on top of the C-ABI.

Mirrors program vac (src/vac.t:5-158): read the parameters (par/DEFAULT values,
then vac.par), read the initial snapshot, set up grid and boundaries, then loop
  save if due -> dt -> stop test -> slowsteps/tmaxexact -> advance -> it, t
with every compute call going to libsacgpu.so.  Snapshots (.out) and the log
(.log) are written in the reference's formats (sac_b200.fileio).

    python -m sac_b200.vac vac.par [--user gravvisc|slog|viscosity|strat|tube|none]
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

from . import abi, fileio, params

# par/DEFAULT (the reference's default parameter file), the keys this driver uses
DEFAULT_PAR = """
 &testlist teststr=' ' /
 &filelist typefileini='auto' typefileout='auto' typefilelog='default'
    snapshotini=0 snapshotout=0 fullgridini=F fullgridout=F /
 &savelist /
 &stoplist itmax=1000000 tmax=1.D99 tmaxexact=F dtmin=1.D-99 residmin=0.D0 residmax=1.D99 /
 &methodlist typeadvance='twostep' dimsplit=T typedimsplit='default' sourcesplit=F sourceunsplit=T
    typesourcesplit='default' divbfix=T smallfix=F compactres=F /
 &boundlist extraB=F /
 &paramlist courantpar=0.8D0 dtcantgrow=F dtdiffpar=0.5D0 dtpar=-1.D0 slowsteps=0 /
"""

BIG, BIGINT, SMALL = 1e99, 10000000, 1e-99
USER = {"none": params.USR_NONE, "viscosity": params.USR_VISCOSITY, "slog": params.USR_SLOG,
        "gravvisc": params.USR_GRAVVISC, "strat": params.USR_STRAT, "tube": params.USR_TUBE}


def _list(v, n, fill):
    if v is None:
        return [fill] * n
    v = v if isinstance(v, list) else [v]
    return (v + [fill] * n)[:n]


def eqpar_map(eqpar, names, ndim):
    """gamma, eta, gravity and nu from eqpar (src/vacpar.t.mhd:26, src/vacusrpar.f:3-6).

    The .ini's variable-name line ends with the eqpar names; when they are present
    they decide, otherwise the reference's positions grav^D_=neqpar+^D+1, nu_=neqpar+4."""
    out = {"gamma": float(eqpar[0]), "eta": float(eqpar[1]) if len(eqpar) > 1 else 0.0,
           "grav": [0.0, 0.0, 0.0], "nu": 0.0}
    nm = [n.lower() for n in names[-len(eqpar):]] if names else []
    if len(nm) == len(eqpar) and nm[:1] == ["gamma"]:
        for v, n in zip(eqpar, nm):
            if n.startswith("grav") and n[4:].isdigit() and 1 <= int(n[4:]) <= 3:
                out["grav"][int(n[4:]) - 1] = float(v)
            elif n == "nu":
                out["nu"] = float(v)
        return out
    for d in range(ndim):
        if 3 + d < len(eqpar):
            out["grav"][d] = float(eqpar[3 + d])
    if len(eqpar) > 5:
        out["nu"] = float(eqpar[5])
    return out


def header_strings(fileheadout, varnames, ndim, ndir, user):
    """setheaderstrings (src/vacio.t:844-898): a headline without '_' gains
    '_mhd<ndim><ndir>'; varnames gains the equation parameter names 'gamma eta'
    and, for the gravity modules, 'grav1 .. grav<ndim>' when missing (the
    Stuart user parameters, sac/src/vacusrpar.t.stuart:10-12).  The reference
    stops when the headline names another configuration than it was built for;
    this library takes its configuration from the file, so it keeps the name."""
    head = fileheadout.rstrip()
    if "_" not in head:
        head = head + "_mhd%d%d" % (ndim, ndir)
    names = varnames.rstrip()
    if names != "default":
        if "gamma eta" not in names:
            names = names + "   gamma eta"
        special = " ".join("grav%d" % (d + 1) for d in range(ndim))
        if user in ("gravvisc", "slog", "strat", "tube") and special not in names:
            names = names + "   " + special
    return head, names


class Run:
    def __init__(self, par_text: str, user: str = "gravvisc", default_text: str = DEFAULT_PAR, device=0,
                 context=None):
        """context: the class behind the C-ABI calls (abi.Context, the device
        library, by default)."""
        pf = params.read_par(default_text, par_text)
        self.pf = pf
        g = lambda grp, k, d=None: pf.get(grp, k, d)  # noqa: E731
        self.filenameini = g("filelist", "filenameini")
        fn = g("filelist", "filename", ["run.log", "run.out"])
        self.filename = fn if isinstance(fn, list) else [fn]
        self.typefileini = g("filelist", "typefileini", "auto")
        self.typefileout = g("filelist", "typefileout", "auto")
        self.snapshotini = int(g("filelist", "snapshotini", 0))
        self.snapshotout = int(g("filelist", "snapshotout", 0))
        self.fullgridini = bool(g("filelist", "fullgridini", False))
        self.fullgridout = bool(g("filelist", "fullgridout", False))
        snap = fileio.read_ini(self.filenameini, self.typefileini, self.snapshotini)
        if self.typefileout == "auto":
            self.typefileout = fileio.detect_type(self.filenameini) if self.typefileini == "auto" else self.typefileini
        self.snap = snap
        ndim = abs(snap.ndim)
        nw = snap.nw
        ndir = (nw - 4) // 3
        if 3 * ndir + 4 != nw:
            raise ValueError(f"nw={nw} is not an MHD variable count")
        self.ndim, self.ndir, self.nw = ndim, ndir, nw
        nx = tuple(snap.nx)
        if self.fullgridini:
            nx = tuple(n - 4 for n in nx)
        self.nx = nx
        self.ixGhi = tuple(n + 4 for n in nx)
        self.ixM = tuple([3] * ndim + [1] * (3 - ndim) + [n + 2 for n in nx] + [1] * (3 - ndim))
        # full-grid x and w
        shape = self.ixGhi
        self.x = np.zeros(shape + (ndim,), order="F")
        self.w = np.zeros(shape + (nw,), order="F")
        sl = tuple(slice(None) if self.fullgridini else slice(2, 2 + n) for n in nx)
        self.x[sl] = snap.x
        self.w[sl] = snap.w
        # stop/save lists
        self.it = int(g("stoplist", "it", snap.it))
        self.t = float(g("stoplist", "t", snap.t))
        self.itmax = int(g("stoplist", "itmax", BIGINT))
        self.tmax = float(g("stoplist", "tmax", BIG))
        self.tmaxexact = bool(g("stoplist", "tmaxexact", False))
        self.dtmin = float(g("stoplist", "dtmin", SMALL))
        # steady-state stop on the residual ||w_n+1 - w_n||, src/vac.t:88-98, 596-597
        self.residmin = float(g("stoplist", "residmin", 0.0))
        self.residmax = float(g("stoplist", "residmax", BIG))
        self.use_residual = self.residmin > 0.0 or self.residmax < BIG
        self.residual = BIG
        # stop once this much CPU time has passed since the start, src/vac.t:599-600
        self.cputimemax = float(g("stoplist", "cputimemax", BIG))
        self.time0 = time.process_time()
        self.dtsave = [float(v) for v in _list(g("savelist", "dtsave"), 2, BIG)]
        self.ditsave = [int(v) for v in _list(g("savelist", "ditsave"), 2, BIGINT)]
        self.tsave = [[BIG], [BIG]]
        self.itsave = [[BIGINT], [BIGINT]]
        for k, v in pf.groups.get("savelist", {}).items():
            if k.startswith("itsave(") or k.startswith("tsave("):
                i, f = (int(a) for a in k[k.index("(") + 1:-1].split(","))
                tgt = self.itsave if k.startswith("itsave") else self.tsave
                while len(tgt[f - 1]) < i:
                    tgt[f - 1].append(BIGINT if tgt is self.itsave else BIG)
                tgt[f - 1][i - 1] = v
        # methods
        typefull = _list(g("methodlist", "typefull"), nw, "nul")
        self.iws = [iw + 1 for iw in range(nw) if typefull[iw] != "nul"]
        self.method = next((t for t in typefull if t != "nul"), "nul")
        typeadvance = g("methodlist", "typeadvance", "twostep")
        typepred = _list(g("methodlist", "typepred"), nw, "default")
        pred = next((p for p in typepred if p != "nul"), "default")
        if pred == "default":
            pred = "nul" if self.method in ("cd4", "cd", "nul") else pred
        if typeadvance == "twostep" and pred == "nul":
            typeadvance = "onestep"  # src/vacio.t:502
        dimsplit = bool(g("methodlist", "dimsplit", True))
        tds = g("methodlist", "typedimsplit", "default")
        if tds == "default":
            tds = "xyyx" if dimsplit else "unsplit"
        self.typedimsplit = tds
        self.dimsplit = tds != "unsplit"
        if bool(g("methodlist", "sourcesplit", False)):
            raise NotImplementedError("sourcesplit=T is outside the implemented path")
        # the Powell source is on by default (par/DEFAULT:46) and needs unsplit
        # sources here, since split sources are not built (src/vacio.t:357-359)
        divbfix = bool(g("methodlist", "divbfix", True))
        sourceunsplit = bool(g("methodlist", "sourceunsplit", True))
        if divbfix and not sourceunsplit:
            raise ValueError("divbfix=T requires unsplitsource=T or splitsource=T !")
        # options that change the run but are not built: say so rather than ignore them
        for grp, key, off, what in (("methodlist", "divbconstrain", False, "divbconstrain=T (the CT module)"),
                                    ("boundlist", "extraB", False, "extraB=T (a user specialbound before every fill)")):
            if bool(g(grp, key, off)) != off:
                raise NotImplementedError(what + " is outside the implemented path")
        if str(g("filelist", "typefilelog", "default")).strip() != "default":
            raise NotImplementedError("typefilelog other than 'default' (savefilelog_special) is not built")
        # &methodlist is read after the initial file, so its eqpar and fileheadout
        # override the file's (src/vacio.t:208-246)
        eqpar = [float(v) for v in snap.eqpar]
        mth = pf.groups.get("methodlist", {})
        if "eqpar" in mth:
            vals = mth["eqpar"] if isinstance(mth["eqpar"], list) else [mth["eqpar"]]
            for i, val in enumerate(vals):
                if i < len(eqpar):
                    eqpar[i] = float(val)
        for k, val in mth.items():
            if k.startswith("eqpar(") and k.endswith(")"):
                i = int(k[6:-1]) - 1
                if 0 <= i < len(eqpar):
                    eqpar[i] = float(val)
        self.eqpar = eqpar
        ep = eqpar_map(eqpar, snap.varnames.split(), ndim)
        self.params = params.make_params(
            gamma=ep["gamma"], eta=ep["eta"], grav=ep["grav"], nu=ep["nu"],
            courantpar=float(g("paramlist", "courantpar", 0.8)), dtpar=float(g("paramlist", "dtpar", -1.0)),
            dtdiffpar=float(g("paramlist", "dtdiffpar", 0.5)), dtcantgrow=int(bool(g("paramlist", "dtcantgrow", False))),
            typeadvance=typeadvance, typepred=pred, sourceunsplit=int(sourceunsplit),
            divbfix=int(divbfix), user=USER[user], device=device,
            # keeppositive's switch and floors, src/vacio.t:44-45,99-101
            smallfix=int(bool(g("methodlist", "smallfix", False))),
            smallp=float(g("methodlist", "smallp", -1.0)), smallrho=float(g("methodlist", "smallrho", -1.0)),
            vacuumrho=float(g("methodlist", "vacuumrho", -1.0)),
            # addsource_res1 instead of addsource_res2 for eta > 0, par/DEFAULT:57
            compactres=int(bool(g("methodlist", "compactres", False))))
        self.slowsteps = int(g("paramlist", "slowsteps", 0))
        if self.slowsteps == 1 and float(g("paramlist", "dtpar", -1.0)) > 0.0:
            # src/vac.t:76 resets dtpar after the first step; the context's
            # parameters are fixed at its creation
            raise NotImplementedError("slowsteps=1 with dtpar>0 is outside the implemented path")
        # &boundlist regions: the default 2*ndim, or the user's ixB^LIM/idimB/upperB
        self.nB, self.regions, self.ipairB = params.boundary_regions_from_par(pf, ndim)
        self.types = params.typeB_from_par(pf, nw, self.nB)
        self.wnames = g("methodlist", "wnames", snap.varnames)
        self.fileheadout, self.varnames = header_strings(str(g("methodlist", "fileheadout", snap.header)),
                                                         snap.varnames, ndim, ndir, user)
        # state of the save logic, src/vac.t:179-184
        self.tsavelast = [self.t, self.t]
        self.itsavelast = [self.it, self.it]
        self.isavet = [0, 0]
        self.isaveit = [0, 0]
        self.isaveout = 0
        self.itmin = self.it
        self.dt = 0.0
        self.ctx = (context or abi.Context)(self.params)
        self.ctx.set_grid(ndim, ndir, self.ixGhi, self.ixM, self.x, self.fullgridini)
        self.ctx.set_boundaries(params.pack_typeB(self.types), self.nB, ipairB=self.ipairB, regions=self.regions)
        self.ctx.upload(self.w)
        self.ctx.getboundary(self.t)

    # -- timetosave, src/vac.t:608-638; savefile, src/vacio.t:901-958 -------------
    def _tsave(self, ifile, k):
        lst = self.tsave[ifile]
        return lst[k] if k < len(lst) else BIG

    def _itsave(self, ifile, k):
        lst = self.itsave[ifile]
        return lst[k] if k < len(lst) else BIGINT

    def timetosave(self, ifile):
        ok = False
        if self.t >= self._tsave(ifile, self.isavet[ifile]):
            ok = True
            self.isavet[ifile] += 1
        if self.it == self._itsave(ifile, self.isaveit[ifile]):
            ok = True
            self.isaveit[ifile] += 1
        if self.it == self.itsavelast[ifile] + self.ditsave[ifile]:
            ok = True
        if self.t >= self.tsavelast[ifile] + self.dtsave[ifile]:
            ok = True
        if ok:
            self.tsavelast[ifile] = self.t
            self.itsavelast[ifile] = self.it
        return ok

    def savefile(self, ifile):
        w = self.ctx.download()
        if ifile == 1:
            base = self.filename[1] if len(self.filename) > 1 else "run.out"
            append = self.out_open
            if self.snapshotout > 0 and self.isaveout > 0 and self.isaveout % self.snapshotout == 0:
                self.outname = f"{base}_{self.isaveout + 1}"
                append = False
            elif self.outname is None:
                self.outname = base
            self.isaveout += 1
            if self.fullgridout:
                xs, ws, nx = self.x, w, self.ixGhi
            else:
                sl = tuple(slice(2, 2 + n) for n in self.nx)
                xs, ws, nx = self.x[sl], w[sl], self.nx
            s = fileio.Snapshot(self.fileheadout, self.it, self.t, self.ndim, len(self.eqpar), self.nw,
                                tuple(nx), np.asarray(self.eqpar), self.varnames, np.asfortranarray(xs),
                                np.asfortranarray(ws))
            if self.typefileout == "ascii":
                fileio.write_ascii(self.outname, s, append=append)
            else:
                fileio.write_binary(self.outname, s, append=append)
            self.out_open = True
        else:
            d = self.ctx.diag()
            name = self.filename[0]
            with open(name, "a" if self.log_open else "w") as f:
                if not self.log_open:
                    fileio.write_log_header(f, self.fileheadout, self.wnames, self.use_residual)
                f.write(fileio.format_log_line(self.it, self.t, self.dt, list(d.wmean)[: self.nw],
                                               self.residual if self.use_residual else None) + "\n")
            self.log_open = True

    outname = None
    out_open = False
    log_open = False

    # -- the main loop, src/vac.t:55-106 ---------------------------------------------
    def timetofinish(self):
        ok = (self.it >= self.itmax or self.t >= self.tmax or self.dt < self.dtmin
              or (self.it > self.itmin and (self.residual < self.residmin or self.residual > self.residmax)))
        if self.cputimemax < BIG and not ok:
            ok = self.cputimemax <= time.process_time() - self.time0
        return ok

    def step(self):
        for ifile in (0, 1):
            if self.timetosave(ifile):
                self.savefile(ifile)
        dt = self.ctx.getdt(self.it)
        self.dt = dt
        if self.timetofinish():
            return False
        if self.slowsteps > self.it - self.itmin + 1:
            # dt*(one-(one-(it-itmin+one)/slowsteps)**2), src/vac.t:79; **2 is a product
            q = 1.0 - (self.it - self.itmin + 1.0) / self.slowsteps
            dt = dt * (1.0 - q * q)
        if self.tmaxexact:
            dt = min(dt, self.tmax - self.t + SMALL)
        self.dt = dt
        wold = self.ctx.download() if self.use_residual else None
        if self.dimsplit and self.ndim > 1:
            order = range(1, self.ndim + 1)
            if not ((self.it // 2) * 2 == self.it or self.typedimsplit == "xy"):
                order = range(self.ndim, 0, -1)
            for d in order:
                self.ctx.advect(dt, self.t, self.it, method=self.method, iws=self.iws, idimmin=d, idimmax=d)
        else:
            self.ctx.advect(dt, self.t, self.it, method=self.method, iws=self.iws)
        if self.use_residual:
            self.residual = self.getresidual(wold, self.ctx.download())
        self.it += 1
        self.t += dt
        return True

    def getresidual(self, wold, w):
        """sqrt(sum over iw of ||w - wold||^2 / ||w||^2 (1 where ||w||^2 < smalldouble)
        / nw) over the mesh, src/vac.t:88-98."""
        sl = tuple(slice(2, 2 + n) for n in self.nx)
        residual = 0.0
        for iw in range(self.nw):
            a, b = w[sl + (iw,)], wold[sl + (iw,)]
            wnrm2 = float((a * a).sum())
            if wnrm2 < SMALL:
                wnrm2 = 1.0
            residual = residual + float(((a - b) * (a - b)).sum()) / wnrm2
        return float(np.sqrt(residual / self.nw))

    def run(self, verbose=True):
        t0 = time.time()
        if verbose:
            print(f"Start Advance {time.time() - t0:10.3f} sec")
        while self.step():
            pass
        for ifile in (0, 1):
            if self.itsavelast[ifile] < self.it:
                self.savefile(ifile)
        if verbose:
            print(f"Finish Advance {time.time() - t0:10.3f} sec   it={self.it} t={self.t:.6g}")
            for line in self.final_report():
                print(line)
        return self

    def final_report(self):
        """What program vac prints after the loop (src/vac.t:117-136): the dtmin and
        cputimemax warnings and, with smallfix, keeppositive's error, first as it
        reports it at the first occurrence (src/vacphys.t.mhd:36-40), then its count."""
        out = []
        if self.dt < self.dtmin:
            out.append(" Warning: dt<dtmin !!!")
        if time.process_time() - self.time0 > self.cputimemax:
            out.append(" Warning: cputimemax exceeded !!!")
        if self.params.smallfix:
            d = self.ctx.diag()
            if d.nerror_toosmallp > 0:
                out.append(f"Too small pressure (code= 1) at it={d.toosmallp_it:7d}")
                out.append(f" Value < smallp:  {d.toosmallp_min!r} {self.params.smallp!r}")
                out.append(f"Error (code= 1) occurred {d.nerror_toosmallp:5d} times !!!")
                out.append("Error description: Pressure below psmall")
        return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("par", help="vac.par")
    ap.add_argument("--user", default="gravvisc", choices=sorted(USER))
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    with open(a.par) as f:
        Run(f.read(), a.user, device=a.device).run()


if __name__ == "__main__":
    sys.exit(main())
