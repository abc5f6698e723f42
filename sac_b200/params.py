"""Parameters of the hot path and the reader of SAC/VAC parameter files.

`SacParams` is the ctypes image of `sac_params` in include/sac_gpu.h.  `read_par`
parses the Fortran NAMELIST groups of `par/DEFAULT` and `vac.par`
(src/vacio.t:25-53, read order src/vacio.t:121-132 then :173-455) for the keys
that the hot path uses; unknown keys are kept verbatim in the returned dict so a
caller can still inspect them.
"""
from __future__ import annotations

import ctypes
import re
from dataclasses import dataclass, field

LENTYPE = 10  # CHARACTER*^LENTYPE, src/vacpp.pl:156
NHIB = 10     # nhiB, src/vacdef.t:34
NWMAX = 13

USR_NONE, USR_VISCOSITY, USR_SLOG, USR_GRAVVISC, USR_STRAT, USR_TUBE = range(6)
PREC_FP64, PREC_FP32 = 0, 1

STATUS = {
    0: "SAC_OK", 1: "SAC_ERR_ARG", 2: "SAC_ERR_STATE", 3: "SAC_ERR_CUDA",
    4: "SAC_ERR_NOMEM", 5: "SAC_ERR_UNSUPPORTED", 6: "SAC_ERR_NONFINITE",
    7: "SAC_ERR_TIMEOUT", 8: "SAC_ERR_NODEVICE",
}


class SacParams(ctypes.Structure):
    _fields_ = [
        ("gamma", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("grav", ctypes.c_double * 3),
        ("nu", ctypes.c_double),
        ("courantpar", ctypes.c_double),
        ("dtpar", ctypes.c_double),
        ("dtdiffpar", ctypes.c_double),
        ("dtcantgrow", ctypes.c_int),
        ("typeadvance", ctypes.c_char * (LENTYPE + 1)),
        ("typepred", ctypes.c_char * (LENTYPE + 1)),
        ("sourceunsplit", ctypes.c_int),
        ("divbfix", ctypes.c_int),
        ("user", ctypes.c_int),
        ("userpar", ctypes.c_double * 16),
        ("alias_nu_grav3", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
        ("smallfix", ctypes.c_int),
        ("smallp", ctypes.c_double),
        ("smallrho", ctypes.c_double),
        ("vacuumrho", ctypes.c_double),
        ("compactres", ctypes.c_int),
    ]


class SacDiag(ctypes.Structure):
    _fields_ = [
        ("wmean", ctypes.c_double * NWMAX),
        ("divb_l2", ctypes.c_double),
        ("divb_linf", ctypes.c_double),
        ("maxviscoef", ctypes.c_double),
        ("ctot", ctypes.c_double * 3),
        ("nonfinite", ctypes.c_int),
        ("nerror_toosmallp", ctypes.c_int),
        ("toosmallp_it", ctypes.c_int),
        ("toosmallp_min", ctypes.c_double),
    ]


def default_params() -> SacParams:
    """par/DEFAULT values for the keys of sac_params (par/DEFAULT:30-86)."""
    p = SacParams()
    p.gamma = 5.0 / 3.0
    p.eta = 0.0
    p.nu = 0.0
    p.courantpar = 0.8
    p.dtpar = -1.0
    p.dtdiffpar = 0.5
    p.dtcantgrow = 0
    p.typeadvance = b"twostep"
    p.typepred = b"nul"
    p.sourceunsplit = 1
    p.divbfix = 0
    p.user = USR_NONE
    p.alias_nu_grav3 = 0
    p.precision = PREC_FP64
    p.device = 0
    p.smallfix = 0  # par/DEFAULT:54
    p.smallp = p.smallrho = p.vacuumrho = -1.0  # src/vacio.t:99-101
    p.compactres = 0  # par/DEFAULT:57
    return p


def make_params(**kw) -> SacParams:
    p = default_params()
    for k, v in kw.items():
        if k == "grav":
            for i, g in enumerate(v):
                p.grav[i] = g
        elif k == "userpar":
            for i, g in enumerate(v):
                p.userpar[i] = g
        elif k in ("typeadvance", "typepred"):
            setattr(p, k, v.encode() if isinstance(v, str) else v)
        else:
            setattr(p, k, v)
    return p


def pack_typeB(types: list[list[str]]) -> bytes:
    """CHARACTER*10 typeB(nw,nB) in Fortran order: types[iB][iw]."""
    out = bytearray()
    for iB_types in types:
        for t in iB_types:
            if len(t) > LENTYPE:
                raise ValueError(f"boundary type {t!r} longer than {LENTYPE}")
            out += t.encode().ljust(LENTYPE, b" ")
    return bytes(out)


# ---------------------------------------------------------------------------
# NAMELIST reader (subset sufficient for SAC par files)
# ---------------------------------------------------------------------------
def _strip_comments(text: str) -> str:
    out = []
    for line in text.splitlines():
        q, cut = None, len(line)
        for i, ch in enumerate(line):
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "!":
                cut = i
                break
        out.append(line[:cut])
    return "\n".join(out)


def _groups(text: str):
    """Yield (name, body) for each &name ... / group, honouring quotes."""
    i, n = 0, len(text)
    while True:
        j = text.find("&", i)
        if j < 0:
            return
        k = j + 1
        while k < n and (text[k].isalnum() or text[k] == "_"):
            k += 1
        name = text[j + 1:k].lower()
        q, m = None, k
        while m < n:
            ch = text[m]
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "/" or (ch == "&" and text[m:m + 4].lower() == "&end"):
                break
            m += 1
        yield name, text[k:m]
        i = m + 1


def _lex(body: str):
    """Tokens: ('key', name) for 'name=' (name may carry an index), ('val', text)."""
    toks, i, n = [], 0, len(body)
    while i < n:
        ch = body[i]
        if ch in " \t\r\n,":
            i += 1
            continue
        if ch in "'\"":
            j = body.find(ch, i + 1)
            j = n if j < 0 else j
            toks.append(("val", body[i:j + 1]))
            i = j + 1
            continue
        j, depth = i, 0
        while j < n:
            c = body[j]
            if c == "(":
                depth += 1
            elif c == ")":
                depth -= 1
            elif depth == 0 and (c in " \t\r\n,=" or c in "'\""):
                break
            j += 1
        word = body[i:j]
        # repeat count followed by a quoted string: 6*'cd4'
        if word.endswith("*") and j < n and body[j] in "'\"":
            q = body[j]
            k = body.find(q, j + 1)
            k = n if k < 0 else k
            toks.append(("val", word + body[j:k + 1]))
            i = k + 1
            continue
        k = j
        while k < n and body[k] in " \t":
            k += 1
        if k < n and body[k] == "=":
            toks.append(("key", word))
            i = k + 1
        else:
            toks.append(("val", word))
            i = j
    return toks


def _value(tok: str):
    t = tok.strip()
    m = re.fullmatch(r"(\d+)\*(.*)", t, re.S)
    if m:
        return [_value(m.group(2))] * int(m.group(1))
    if t[:1] in "'\"":
        return t[1:-1]
    tl = t.lower()
    if tl in (".true.", "t", ".t."):
        return True
    if tl in (".false.", "f", ".f."):
        return False
    try:
        if re.fullmatch(r"[+-]?\d+", t):
            return int(t)
        return float(tl.replace("d", "e"))
    except ValueError:
        return t


def parse_namelists(text: str) -> dict[str, dict]:
    """Parse Fortran NAMELIST groups into {group: {key: value-or-list}}.

    Array element keys such as itsave(1,2) keep their index text."""
    groups: dict[str, dict] = {}
    for name, body in _groups(_strip_comments(text)):
        vals: dict = {}
        key = None
        for kind, tok in _lex(body):
            if kind == "key":
                key = tok.strip().lower()
                vals[key] = []
            elif key is not None:
                v = _value(tok)
                if isinstance(v, list):
                    vals[key].extend(v)
                else:
                    vals[key].append(v)
        for k, v in list(vals.items()):
            vals[k] = v[0] if len(v) == 1 else v
        groups.setdefault(name, {}).update(vals)
    return groups


@dataclass
class ParFile:
    """Merged view of par/DEFAULT followed by vac.par (later values win)."""

    groups: dict = field(default_factory=dict)

    def get(self, group: str, key: str, default=None):
        return self.groups.get(group, {}).get(key.lower(), default)


def read_par(*texts: str) -> ParFile:
    pf = ParFile()
    for t in texts:
        for g, vals in parse_namelists(t).items():
            pf.groups.setdefault(g, {}).update(vals)
    return pf


def typeB_from_par(pf: ParFile, nw: int, nB: int) -> list[list[str]]:
    """typeB(nw,nB) from &boundlist (column-major fill as NAMELIST does)."""
    raw = pf.get("boundlist", "typeb", "cont")
    flat = raw if isinstance(raw, list) else [raw]
    types = [["cont"] * nw for _ in range(nB)]  # src/vacio.t:104-108
    for n, t in enumerate(flat[: nw * nB]):
        types[n // nw][n % nw] = str(t).strip()
    return types


def _namelist_array(pf: ParFile, group: str, name: str, shape: tuple, default):
    """A NAMELIST array of `shape` (Fortran order) from a whole-array list
    (name = v1, v2, ...) and/or element keys (name(i,j) = v, ...), a list after an
    element key continuing in column-major order, as NAMELIST input fills it."""
    n = 1
    for e in shape:
        n *= e
    flat = [default] * n
    grp = pf.groups.get(group, {})

    def put(start, vals):
        vals = vals if isinstance(vals, list) else [vals]
        for k, v in enumerate(vals):
            if start + k < n:
                flat[start + k] = v

    name = name.lower()
    if name in grp:
        put(0, grp[name])
    for k, v in grp.items():
        if k.startswith(name + "(") and k.endswith(")"):
            idx = [int(x) - 1 for x in k[len(name) + 1:-1].split(",")]
            lin, mul = 0, 1
            for i, e in zip(idx, shape):
                lin += i * mul
                mul *= e
            put(lin, v)
    return flat


def boundary_regions_from_par(pf: ParFile, ndim: int):
    """&boundlist's nB and, when the user gave regions (ixBmax(1,1) /= 0,
    src/vacio.t:117 and src/vacgrid.t:53), (ixBmin, ixBmax, idimB, upperB) as
    Context.set_boundaries takes them, with ipairB (0 = automatic); else None."""
    nB = int(pf.get("boundlist", "nb", 2 * ndim))
    lo = _namelist_array(pf, "boundlist", "ixbmin", (ndim, 10), 0)
    hi = _namelist_array(pf, "boundlist", "ixbmax", (ndim, 10), 0)
    ipair = [int(v) for v in _namelist_array(pf, "boundlist", "ipairb", (10,), 0)][:nB]
    if int(hi[0]) == 0:
        return nB, None, ipair
    idim = [int(v) for v in _namelist_array(pf, "boundlist", "idimb", (10,), 0)][:nB]
    upper = [bool(v) for v in _namelist_array(pf, "boundlist", "upperb", (10,), False)][:nB]
    ixlo = [[int(lo[d + ndim * iB]) for d in range(ndim)] for iB in range(nB)]
    ixhi = [[int(hi[d + ndim * iB]) for d in range(ndim)] for iB in range(nB)]
    return nB, (ixlo, ixhi, idim, upper), ipair
