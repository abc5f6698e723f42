"""ctypes binding of the C-ABI declared in include/sac_gpu.h.

The same binder serves the product library (libsacgpu.so, prefix ``sac_``) and
any library with the identical call shape under another prefix.  It is the Python
counterpart of the ISO_C_BINDING interface a Fortran host would declare.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import STATUS, SacDiag, SacParams

HERE = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIB = os.path.join(HERE, "libsacgpu.so")

# every entry point of include/sac_gpu.h
ABI_SYMBOLS = (
    "default_params", "create", "set_grid", "set_boundaries", "upload", "download",
    "getboundary", "getdt", "advect", "diag", "synchronize", "last_error", "destroy",
)


class SacError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_LIBS: dict = {}


def load(path: str = PRODUCT_LIB, prefix: str = "sac_"):
    key = (os.path.abspath(path), prefix)
    if key in _LIBS:
        return _LIBS[key]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    f = lambda n: getattr(lib, prefix + n)  # noqa: E731
    f("create").argtypes = [ctypes.POINTER(SacParams), ctypes.POINTER(P)]
    f("set_grid").argtypes = [P, ctypes.c_int, ctypes.c_int, ip, ip, dp, ctypes.c_int]
    f("set_boundaries").argtypes = [P, ctypes.c_int, ctypes.c_char_p, ip, ip, ip, ip]
    f("upload").argtypes = [P, dp]
    f("download").argtypes = [P, dp]
    f("getboundary").argtypes = [P, ctypes.c_double]
    f("getdt").argtypes = [P, dp, ctypes.c_int]
    f("advect").argtypes = [P, ctypes.c_char_p, ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                            ctypes.c_double, ctypes.c_int]
    f("diag").argtypes = [P, ctypes.POINTER(SacDiag)]
    f("last_error").argtypes = [P]
    f("last_error").restype = ctypes.c_char_p
    f("destroy").argtypes = [P]
    f("destroy").restype = None
    for n in ("create", "set_grid", "set_boundaries", "upload", "download", "getboundary", "getdt",
              "advect", "diag"):
        f(n).restype = ctypes.c_int
    try:
        f("synchronize").argtypes = [P]
        f("synchronize").restype = ctypes.c_int
    except AttributeError:
        pass
    _LIBS[key] = (lib, prefix)
    return _LIBS[key]


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Context:
    """One resident state behind the C-ABI (sac_create ... sac_destroy)."""

    def __init__(self, params: SacParams, path: str = PRODUCT_LIB, prefix: str = "sac_"):
        self.lib, self.prefix = load(path, prefix)
        self.h = ctypes.c_void_p()
        self._call("create", ctypes.byref(params), ctypes.byref(self.h), ctx=False)
        self.nw = None
        self.shape = None

    def _call(self, name, *args, ctx=True):
        fn = getattr(self.lib, self.prefix + name)
        st = fn(self.h, *args) if ctx else fn(*args)
        if st != 0:
            msg = getattr(self.lib, self.prefix + "last_error")(self.h) if self.h else b""
            raise SacError(st, f"{self.prefix}{name}: {(msg or b'').decode(errors='replace')}")
        return st

    def set_grid(self, ndim, ndir, ixGhi, ixM, x, fullgridini=False):
        ixGhi = np.ascontiguousarray(list(ixGhi) + [1] * (3 - len(ixGhi)), dtype=np.int32)
        ixM = np.ascontiguousarray(ixM, dtype=np.int32)
        x = np.asfortranarray(x, dtype=np.float64)
        self._call("set_grid", int(ndim), int(ndir), _ip(ixGhi), _ip(ixM),
                   _dp(x.reshape(-1, order="F")), int(bool(fullgridini)))
        self.nw = 3 * ndir + 4
        self.shape = tuple(int(v) for v in ixGhi[:ndim])

    def set_boundaries(self, typeB_packed: bytes, nB: int, ipairB=None, regions=None):
        """boundsetup.  regions: None for the default 2*ndim regions, or the user's
        as (ixBmin, ixBmax, idimB, upperB): ixBmin/ixBmax [nB][ndim] 1-based
        inclusive limits, idimB [nB] in 1..ndim, upperB [nB] booleans."""
        keep = []

        def arr(v):
            a = np.ascontiguousarray(v, dtype=np.int32).reshape(-1)
            keep.append(a)
            return _ip(a)

        ip = arr(ipairB) if ipairB is not None else None
        ixb = idb = upb = None
        if regions is not None:
            lo, hi, idim, upper = regions
            ixb = arr(np.concatenate([np.asarray(lo, dtype=np.int32).reshape(-1),
                                      np.asarray(hi, dtype=np.int32).reshape(-1)]))
            idb = arr(idim)
            upb = arr([1 if u else 0 for u in upper])
        self._keep = keep
        self._call("set_boundaries", int(nB), typeB_packed, ixb, idb, upb, ip)

    def upload(self, w):
        w = np.asfortranarray(w, dtype=np.float64)
        self._call("upload", _dp(w.reshape(-1, order="F")))

    def download(self, out=None):
        if out is None:
            out = np.empty(self.shape + (self.nw,), dtype=np.float64, order="F")
        self._call("download", _dp(out.reshape(-1, order="F")))
        return out

    def getboundary(self, t=0.0):
        self._call("getboundary", float(t))

    def getdt(self, it):
        dt = ctypes.c_double(0.0)
        self._call("getdt", ctypes.byref(dt), int(it))
        return dt.value

    def advect(self, dt, t, it, method="cd4", iws=None, idimmin=1, idimmax=None):
        ndim = len(self.shape)
        if idimmax is None:
            idimmax = ndim
        ip = None
        if iws is not None:
            arr = np.zeros(self.nw + 1, dtype=np.int32)
            arr[: len(iws)] = iws
            arr[self.nw] = len(iws)
            self._iws = arr
            ip = _ip(arr)
        self._call("advect", method.encode(), ip, int(idimmin), int(idimmax), float(dt), float(t), int(it))

    def diag(self):
        d = SacDiag()
        self._call("diag", ctypes.byref(d))
        return d

    def synchronize(self):
        fn = getattr(self.lib, self.prefix + "synchronize", None)
        if fn is not None:
            self._call("synchronize")

    def close(self):
        if self.h:
            getattr(self.lib, self.prefix + "destroy")(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
