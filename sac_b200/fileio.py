"""SAC/VAC snapshot files: .ini/.out in ASCII and Fortran-unformatted binary.

Record layout follows savefileout_asc / savefileout_bin and their readers
(src/vacio.t:591-752, :961-1091):

    fileheadout                        CHARACTER*400 (binary) / one line (ASCII)
    it, t, ndim, neqpar+nspecialpar, nw   i4, r8, i4, i4, i4
    nx(1:ndim)                         i4
    eqpar(1:neqpar+nspecialpar)        r8
    varnames                           CHARACTER*400 (binary) / one line (ASCII)
    x(ix^S, 1:ndim)                    one record, x1 fastest, then idim
    w(ix^S, iw)                        one record per variable (binary);
                                       ASCII: one row per cell: x(1:ndim), w(1:nw)

Binary records are Fortran sequential-unformatted with 4-byte length markers
before and after each record.  A file holds one or more snapshots appended.
ASCII rows use (100(1pe18.10)) with |w|<=5e-16 written as 0
(src/vacio.t:989-997); the header lines use (i7,1pe13.5,3i3), (3i4) and
(100(1pe13.5)).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

LENNAME = 400  # CHARACTER*^LENNAME, src/vacpp.pl:157


@dataclass
class Snapshot:
    header: str
    it: int
    t: float
    ndim: int          # negative for generalised coordinates
    neqpar: int
    nw: int
    nx: tuple
    eqpar: np.ndarray
    varnames: str
    x: np.ndarray      # shape nx + (ndim,), Fortran order in memory
    w: np.ndarray      # shape nx + (nw,), Fortran order in memory
    extra: dict = field(default_factory=dict)


# ---------------------------------------------------------------------------
# Fortran formatting helpers
# ---------------------------------------------------------------------------
def _fmt_1pe(v: float, width: int, digits: int) -> str:
    """Fortran 1PEw.d: one digit before the point, exponent Esxx."""
    if not np.isfinite(v):
        s = "NaN" if np.isnan(v) else ("Infinity" if v > 0 else "-Infinity")
        return s.rjust(width)
    if v == 0.0:
        mant, exp = 0.0, 0
    else:
        exp = int(np.floor(np.log10(abs(v))))
        mant = v / 10.0 ** exp
        # rounding may carry into a new decade
        r = round(abs(mant), digits)
        if r >= 10.0:
            exp += 1
            mant = v / 10.0 ** exp
    s = f"{mant:.{digits}f}E{exp:+03d}"
    return s.rjust(width)


def _fmt_i(v: int, width: int) -> str:
    s = str(int(v))
    return s.rjust(width) if len(s) <= width else "*" * width


def format_header_line(it, t, ndim, neqpar, nw) -> str:
    # (i7,1pe13.5,3i3)
    return _fmt_i(it, 7) + _fmt_1pe(t, 13, 5) + _fmt_i(ndim, 3) + _fmt_i(neqpar, 3) + _fmt_i(nw, 3)


def format_nx_line(nx) -> str:
    # (3i4): more than three values wrap onto new lines
    parts = [_fmt_i(n, 4) for n in nx]
    return "\n".join("".join(parts[i:i + 3]) for i in range(0, len(parts), 3))


def format_reals(vals, width, digits, per_line=100) -> str:
    parts = [_fmt_1pe(float(v), width, digits) for v in vals]
    return "\n".join("".join(parts[i:i + per_line]) for i in range(0, len(parts), per_line))


# ---------------------------------------------------------------------------
# ASCII
# ---------------------------------------------------------------------------
def write_ascii(path, snaps, append=False):
    mode = "a" if append else "w"
    with open(path, mode) as f:
        for s in snaps if isinstance(snaps, (list, tuple)) else [snaps]:
            f.write(s.header.rstrip() + "\n")
            f.write(format_header_line(s.it, s.t, s.ndim, s.neqpar, s.nw) + "\n")
            f.write(format_nx_line(s.nx) + "\n")
            f.write(format_reals(s.eqpar, 13, 5) + "\n")
            f.write(s.varnames.rstrip() + "\n")
            nd = abs(s.ndim)
            xs = s.x.reshape((-1, nd), order="F")
            ws = s.w.reshape((-1, s.nw), order="F")
            wq = np.where(np.abs(ws) > 5.0e-16, ws, 0.0)
            rows = np.concatenate([xs, wq], axis=1)
            for row in rows:
                f.write(format_reals(row, 18, 10) + "\n")


def read_ascii(path) -> list[Snapshot]:
    """All snapshots of an ASCII .ini/.out file (list-directed reads)."""
    snaps = []
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    while i < len(lines):
        if not lines[i].strip() and i == len(lines) - 1:
            break
        header = lines[i]
        i += 1
        it, t, ndim, neqpar, nw = lines[i].split()[:5]
        it, t, ndim, neqpar, nw = int(it), float(t.replace("D", "E")), int(ndim), int(neqpar), int(nw)
        i += 1
        nd = abs(ndim)
        vals = []
        while len(vals) < nd:
            vals += [int(v) for v in lines[i].split()]
            i += 1
        nx = tuple(vals[:nd])
        vals = []
        while len(vals) < neqpar:
            vals += [float(v.replace("D", "E")) for v in lines[i].split()]
            i += 1
        eqpar = np.array(vals[:neqpar])
        varnames = lines[i]
        i += 1
        ncell = int(np.prod(nx))
        ncol = nd + nw
        data = []
        while len(data) < ncell * ncol:
            data += [float(v.replace("D", "E")) for v in lines[i].split()]
            i += 1
        arr = np.array(data[: ncell * ncol]).reshape(ncell, ncol)
        x = np.asfortranarray(arr[:, :nd].reshape(nx + (nd,), order="F"))
        w = np.asfortranarray(arr[:, nd:].reshape(nx + (nw,), order="F"))
        snaps.append(Snapshot(header, it, t, ndim, neqpar, nw, nx, eqpar, varnames, x, w))
    return snaps


# ---------------------------------------------------------------------------
# binary (Fortran sequential unformatted, 4-byte markers, little endian)
# ---------------------------------------------------------------------------
def _rec(payload: bytes) -> bytes:
    n = struct.pack("<i", len(payload))
    return n + payload + n


def write_binary(path, snaps, append=False):
    mode = "ab" if append else "wb"
    with open(path, mode) as f:
        for s in snaps if isinstance(snaps, (list, tuple)) else [snaps]:
            f.write(_rec(s.header.encode().ljust(LENNAME, b" ")[:LENNAME]))
            f.write(_rec(struct.pack("<idiii", s.it, s.t, s.ndim, s.neqpar, s.nw)))
            f.write(_rec(struct.pack("<" + "i" * len(s.nx), *s.nx)))
            f.write(_rec(np.asarray(s.eqpar, dtype="<f8").tobytes()))
            f.write(_rec(s.varnames.encode().ljust(LENNAME, b" ")[:LENNAME]))
            nd = abs(s.ndim)
            f.write(_rec(np.asarray(s.x, dtype="<f8").reshape(-1, order="F").tobytes()))
            wf = np.asarray(s.w, dtype="<f8").reshape((-1, s.nw), order="F")
            for iw in range(s.nw):
                f.write(_rec(wf[:, iw].tobytes()))
            del nd


def _read_rec(buf: bytes, pos: int):
    (n,) = struct.unpack_from("<i", buf, pos)
    payload = buf[pos + 4: pos + 4 + n]
    (n2,) = struct.unpack_from("<i", buf, pos + 4 + n)
    if n2 != n:
        raise ValueError(f"corrupt record at byte {pos}: markers {n} != {n2}")
    return payload, pos + 8 + n


def read_binary(path) -> list[Snapshot]:
    with open(path, "rb") as f:
        buf = f.read()
    pos, snaps = 0, []
    while pos < len(buf):
        h, pos = _read_rec(buf, pos)
        r, pos = _read_rec(buf, pos)
        it, t, ndim, neqpar, nw = struct.unpack("<idiii", r[:24])
        r, pos = _read_rec(buf, pos)
        nd = abs(ndim)
        nx = struct.unpack("<" + "i" * nd, r[: 4 * nd])
        r, pos = _read_rec(buf, pos)
        eqpar = np.frombuffer(r, dtype="<f8", count=neqpar).copy()
        vn, pos = _read_rec(buf, pos)
        r, pos = _read_rec(buf, pos)
        ncell = int(np.prod(nx))
        x = np.frombuffer(r, dtype="<f8", count=ncell * nd).reshape(nx + (nd,), order="F").copy(order="F")
        w = np.empty(nx + (nw,), order="F")
        for iw in range(nw):
            r, pos = _read_rec(buf, pos)
            w[..., iw] = np.frombuffer(r, dtype="<f8", count=ncell).reshape(nx, order="F")
        snaps.append(Snapshot(h.decode(errors="replace"), it, t, ndim, neqpar, nw, tuple(nx), eqpar,
                              vn.decode(errors="replace"), x, w))
    return snaps


def detect_type(path) -> str:
    """readfileini's auto detection (src/vacio.t:548-564)."""
    with open(path, "rb") as f:
        head = f.read(91).ljust(91, b"\0")
    if head[0] and head[1] and head[2] and head[3]:
        return "ascii"
    if head[88] == 0 and head[89] == 0 and (head[87] == 24 or head[90] == 24):
        return "binary"
    return "special"


def read_snapshots(path, typefileini="auto") -> list[Snapshot]:
    t = detect_type(path) if typefileini == "auto" else typefileini
    if t == "ascii":
        return read_ascii(path)
    if t == "binary":
        return read_binary(path)
    raise ValueError(f"Error in VAC: Unknown typefileini={t}")


def read_ini(path, typefileini="auto", snapshotini=0) -> Snapshot:
    """Last snapshot, or snapshot number snapshotini (1-based) as readfileini does."""
    snaps = read_snapshots(path, typefileini)
    if not snaps:
        raise ValueError(f"no snapshot in {path}")
    if snapshotini > 0:
        return snaps[min(snapshotini, len(snaps)) - 1]
    return snaps[-1]


def write_log_header(f, fileheadout: str, wnames: str, residual: bool):
    """savefilelog_default's header (src/vacio.t:1119-1128)."""
    f.write(fileheadout.rstrip() + "\n")
    if residual:
        f.write("it   t   dt    " + wnames.ljust(55)[:55] + " residual\n")
    else:
        f.write("it   t   dt    " + wnames.ljust(64)[:64] + "\n")


def format_log_line(it, t, dt, wmean, residual=None) -> str:
    # (i7,100(1pe13.5))
    vals = [t, dt] + list(wmean) + ([residual] if residual is not None else [])
    return _fmt_i(it, 7) + format_reals(vals, 13, 5, per_line=100)
