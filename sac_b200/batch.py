"""Many independent 1D/2D problems advanced together (sac_batch_* of libsacgpu.so).

Every instance is its own program-vac run (RK4 'fourstep', its own dt from the
dt block of src/vac.t:60-70); the batch shares one parameter set and one typeB.
Host arrays are the instances' Fortran-order blocks concatenated in instance
order: x(ixG^T,ndim) for the grid, w(ixG^T,nw) for the state.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import abi
from .params import SacParams, make_params, pack_typeB
from .problems import DIXB, make_grid, var_index

P = ctypes.c_void_p
DP = ctypes.POINTER(ctypes.c_double)
IP = ctypes.POINTER(ctypes.c_int)


def _bind(lib):
    if getattr(lib, "_sac_batch_bound", False):
        return lib
    f = lambda n: getattr(lib, "sac_batch_" + n)  # noqa: E731
    f("create").argtypes = [ctypes.POINTER(SacParams), ctypes.c_int, ctypes.c_int, ctypes.c_int, IP,
                            ctypes.c_long, ctypes.POINTER(P)]
    f("set_grid").argtypes = [P, DP]
    f("set_boundaries").argtypes = [P, ctypes.c_char_p]
    f("upload").argtypes = [P, DP]
    f("download").argtypes = [P, DP]
    f("upload_range").argtypes = [P, ctypes.c_int, ctypes.c_int, DP]
    f("download_range").argtypes = [P, ctypes.c_int, ctypes.c_int, DP]
    f("getboundary").argtypes = [P]
    f("advance").argtypes = [P, ctypes.c_int]
    f("state").argtypes = [P, DP, DP, IP]
    f("synchronize").argtypes = [P]
    f("get_stream").argtypes = [P]
    f("get_stream").restype = ctypes.c_void_p
    f("tune").argtypes = [P, IP, DP]
    f("set_driver").argtypes = [P, DP, DP]
    f("set_time").argtypes = [P, DP, IP]
    f("set_tmax").argtypes = [P, DP]
    f("set_stage").argtypes = [P, ctypes.c_int, ctypes.c_int]
    f("get_stage").argtypes = [P, IP, IP, DP, DP]
    f("join").argtypes = [P, P]
    f("unjoin").argtypes = [P]
    f("set_join_form").argtypes = [P, ctypes.c_int]
    f("get_join").argtypes = [P, IP, DP, DP]
    f("mesh_cells").argtypes = [P]
    f("mesh_cells").restype = ctypes.c_long
    f("gather").argtypes = [P, ctypes.c_void_p, ctypes.c_int]
    f("scatter").argtypes = [P, ctypes.c_void_p, ctypes.c_int]
    f("last_error").argtypes = [P]
    f("last_error").restype = ctypes.c_char_p
    f("destroy").argtypes = [P]
    f("destroy").restype = None
    for n in ("create", "set_grid", "set_boundaries", "upload", "download", "upload_range", "download_range",
              "getboundary", "advance", "state", "synchronize", "tune", "set_driver", "set_time", "set_tmax", "gather",
              "scatter", "set_stage", "get_stage", "join", "unjoin", "set_join_form",
              "get_join"):
        f(n).restype = ctypes.c_int
    lib._sac_batch_bound = True
    return lib


def _dp(a):
    return a.ctypes.data_as(DP)


class Batch:
    """ninst instances of mesh sizes nx[i] (tuple of ndim ints each)."""

    def __init__(self, params: SacParams, ndim: int, ndir: int, nx, group_cells: int = 0,
                 path: str = abi.PRODUCT_LIB):
        lib, _ = abi.load(path, "sac_")
        self.lib = _bind(lib)
        self.ndim, self.ndir, self.nw = ndim, ndir, 3 * ndir + 4
        self.nx = [tuple(int(v) for v in n) for n in nx]
        self.ninst = len(self.nx)
        arr = np.ascontiguousarray(np.array(self.nx, dtype=np.int32).reshape(-1))
        self.h = P()
        self._call("create", ctypes.byref(params), ndim, ndir, self.ninst, arr.ctypes.data_as(IP),
                   int(group_cells), ctypes.byref(self.h), own=False)
        self.ncell = [int(np.prod([n + 2 * DIXB for n in s])) for s in self.nx]
        self.woff = np.concatenate([[0], np.cumsum([c * self.nw for c in self.ncell])]).astype(np.int64)

    def _call(self, name, *args, own=True):
        fn = getattr(self.lib, "sac_batch_" + name)
        st = fn(self.h, *args) if own else fn(*args)
        if st != 0:
            msg = self.lib.sac_batch_last_error(self.h) if self.h else b""
            raise abi.SacError(st, f"sac_batch_{name}: {(msg or b'').decode(errors='replace')}")
        return st

    @property
    def mesh_cells(self):
        return int(sum(int(np.prod(s)) for s in self.nx))

    def set_grid(self, x_concat):
        x = np.ascontiguousarray(x_concat, dtype=np.float64)
        self._call("set_grid", _dp(x))

    def set_boundaries(self, typeB):
        self._call("set_boundaries", pack_typeB(typeB))

    def upload(self, w_concat, i0=0, n=None):
        n = self.ninst - i0 if n is None else n
        w = np.ascontiguousarray(w_concat, dtype=np.float64)
        assert w.size == self.woff[i0 + n] - self.woff[i0]
        self._call("upload_range", int(i0), int(n), _dp(w))

    def download(self, i0=0, n=None):
        n = self.ninst - i0 if n is None else n
        out = np.empty(int(self.woff[i0 + n] - self.woff[i0]), dtype=np.float64)
        self._call("download_range", int(i0), int(n), _dp(out))
        return out

    def instance(self, w_concat, i, i0=0):
        """w(ixG^T,nw) of instance i out of a concatenated array starting at instance i0."""
        a = w_concat[self.woff[i] - self.woff[i0]: self.woff[i + 1] - self.woff[i0]]
        shape = tuple(v + 2 * DIXB for v in self.nx[i]) + (self.nw,)
        return a.reshape(shape, order="F")

    def getboundary(self):
        self._call("getboundary")

    def advance(self, nsteps):
        self._call("advance", int(nsteps))

    def state(self):
        t = np.zeros(self.ninst)
        dt = np.zeros(self.ninst)
        it = np.zeros(self.ninst, dtype=np.int32)
        self._call("state", _dp(t), _dp(dt), it.ctypes.data_as(IP))
        return t, dt, it

    def synchronize(self):
        self._call("synchronize")

    def stream(self):
        return self.lib.sac_batch_get_stream(self.h)

    def set_driver(self, A=None, omega=None):
        """Per-instance amplitude and angular frequency of the Gaussian driver."""
        a = None if A is None else np.ascontiguousarray(A, dtype=np.float64)
        o = None if omega is None else np.ascontiguousarray(omega, dtype=np.float64)
        self._call("set_driver", _dp(a) if a is not None else None, _dp(o) if o is not None else None)

    def set_time(self, t=None, it=None):
        ta = None if t is None else np.ascontiguousarray(t, dtype=np.float64)
        ia = None if it is None else np.ascontiguousarray(it, dtype=np.int32)
        self._call("set_time", _dp(ta) if ta is not None else None,
                   ia.ctypes.data_as(IP) if ia is not None else None)

    def set_tmax(self, tmax):
        """Per-instance end time (tmaxexact); <= 0 removes the limit."""
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(tmax, dtype=np.float64), (self.ninst,)))
        self._call("set_tmax", _dp(a))

    def advance_to(self, tmax, chunk=8, max_steps=100000):
        """Advance every instance with its own dt until it lands on tmax; returns
        the largest step count an instance took."""
        self.set_tmax(tmax)
        t0, _, it0 = self.state()
        target = np.broadcast_to(np.asarray(tmax, dtype=np.float64), (self.ninst,))
        done = 0
        while done < max_steps:
            self.advance(chunk)
            done += chunk
            t, _, it = self.state()
            if np.all(t >= target):
                return int((it - it0).max())
        raise RuntimeError("advance_to: tmax not reached")

    PACK = {"f32": 0, "bf16": 1, "f64": 2}

    def gather(self, dev_ptr: int, dtype="f32"):
        """Advanced variables on every instance's mesh into a packed device buffer
        (np*mesh_i values per instance, variable-major, x1 fastest); asynchronous
        on the batch stream."""
        self._call("gather", ctypes.c_void_p(int(dev_ptr)), self.PACK[dtype])

    def scatter(self, dev_ptr: int, dtype="f32"):
        """The reverse of gather; refill the ghosts with getboundary() afterwards."""
        self._call("scatter", ctypes.c_void_p(int(dev_ptr)), self.PACK[dtype])

    @property
    def packed_size(self):
        return int(self.lib.sac_batch_mesh_cells(self.h)) * (2 * self.ndir + 2)

    def tune(self):
        tile = np.zeros(2, dtype=np.int32)
        ms = ctypes.c_double(0.0)
        self._call("tune", tile.ctypes.data_as(IP), ctypes.byref(ms))
        return (int(tile[0]), int(tile[1])), ms.value

    def set_stage(self, fused, shape=0):
        """Each RK stage as the fused per-tile kernel (2D, default sources) in tile
        shape `shape` (0: 32x8, 1: 16x8), or as the face / setnu / update passes."""
        self._call("set_stage", int(bool(fused)), int(shape))

    def stage(self):
        """(fused, shape, ms of one three-pass stage, ms of one fused stage) as the
        tuner measured them (0 before tune)."""
        f, sh = ctypes.c_int(0), ctypes.c_int(0)
        a, b = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self._call("get_stage", ctypes.byref(f), ctypes.byref(sh), ctypes.byref(a), ctypes.byref(b))
        return bool(f.value), sh.value, a.value, b.value

    def join(self, partner):
        """Advance `partner` (FP32 instances, the same parameters) with this FP64
        batch: from now on advance() steps both in one graph, in the faster of
        the two join forms (0: joint kernels over the tiles of both batches, 1:
        each batch's kernels on a branch of its own)."""
        self._call("join", self.h, partner.h, own=False)

    def set_join_form(self, form):
        self._call("set_join_form", int(form))

    def join_info(self):
        """(form, ms of one joint-kernel stage, ms of one two-branch stage)."""
        f = ctypes.c_int(0)
        a, b = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self._call("get_join", ctypes.byref(f), ctypes.byref(a), ctypes.byref(b))
        return f.value, a.value, b.value

    def unjoin(self):
        """End join(): each batch advances alone again."""
        self._call("unjoin")

    def close(self):
        if self.h:
            self.lib.sac_batch_destroy(self.h)
            self.h = P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Orszag-Tang-type vortices of uneven sizes
# ---------------------------------------------------------------------------
OT_SIZES = tuple(range(64, 513, 32))  # {64, 96, ..., 512}


def ot_sizes(ninst, seed=0, sizes=OT_SIZES):
    """nx and ny drawn independently from `sizes` for each instance (seeded)."""
    rng = np.random.default_rng(seed)
    return [(int(a), int(b)) for a, b in zip(rng.choice(sizes, ninst), rng.choice(sizes, ninst))]


def ot_betas(ninst, seed=0, lo=0.5, hi=10.0):
    """Plasma beta of each instance, uniform in [lo, hi] (seeded)."""
    return np.random.default_rng(seed + 7919).uniform(lo, hi, ninst)


class _OTTemplate:
    """The beta-independent part of an Orszag-Tang state on an (nx, ny) grid."""

    def __init__(self, n, gamma, B0):
        self.x = make_grid(n, (0.0, 0.0), (1.0, 1.0))
        X, Y = self.x[..., 0], self.x[..., 1]
        v = var_index(2)
        self.w = np.zeros(X.shape + (v["nw"],), order="F")
        rho = gamma ** 2 * np.ones_like(X)
        vx, vy = -np.sin(2 * math.pi * Y), np.sin(2 * math.pi * X)
        bx, by = B0 * -np.sin(2 * math.pi * Y), B0 * np.sin(4 * math.pi * X)
        self.w[..., v["rho"]] = rho
        self.w[..., v["m0"] + 1] = rho * vx
        self.w[..., v["m0"] + 2] = rho * vy
        self.w[..., v["b0"] + 1] = bx
        self.w[..., v["b0"] + 2] = by
        # kept apart so that e rounds exactly as orszag_tang's p/(g-1) + kin + mag
        self.kin = 0.5 * rho * (vx ** 2 + vy ** 2)
        self.mag = 0.5 * (bx ** 2 + by ** 2)
        self.e = v["e"]


def ot_params(gamma=5.0 / 3.0, nu=1.0, courantpar=0.8, precision=0, dtcantgrow=False):
    """Hyperdiffusion with both dt limits of the gravity/viscosity module and zero
    gravity: the viscous limit (getdt_visc) keeps the supersonic low-beta vortices
    stable at courantpar 0.8, which the Courant limit alone does not."""
    from .params import USR_GRAVVISC
    return make_params(gamma=gamma, nu=nu, courantpar=courantpar, typeadvance="fourstep",
                       user=USR_GRAVVISC, grav=(0.0, 0.0, 0.0), precision=precision,
                       dtcantgrow=int(bool(dtcantgrow)))


class OTBatch:
    """Generator of the uneven Orszag-Tang batch: rho=gamma^2, v=(-sin2pi y,
    sin2pi x), B=B0(-sin2pi y, sin4pi x), p = beta <B^2>/2 with <B^2>=B0^2,
    zero background, periodic boundaries, one beta per instance."""

    def __init__(self, ninst, seed=0, sizes=OT_SIZES, gamma=5.0 / 3.0, B0=1.0, nx=None, betas=None):
        self.nx = list(nx) if nx is not None else ot_sizes(ninst, seed, sizes)
        self.ninst = len(self.nx)
        self.beta = np.asarray(betas) if betas is not None else ot_betas(self.ninst, seed)
        self.gamma, self.B0 = gamma, B0
        self._tpl = {}

    def _template(self, n):
        if n not in self._tpl:
            self._tpl[n] = _OTTemplate(n, self.gamma, self.B0)
        return self._tpl[n]

    def typeB(self):
        return [["periodic"] * 10 for _ in range(4)]

    def x_concat(self):
        return np.concatenate([self._template(n).x.reshape(-1, order="F") for n in self.nx])

    def state(self, i):
        t = self._template(self.nx[i])
        w = t.w.copy(order="F")
        p = self.beta[i] * (self.B0 * self.B0) / 2.0
        w[..., t.e] = p / (self.gamma - 1) + t.kin + t.mag
        return w

    def w_concat(self, i0=0, n=None):
        n = self.ninst - i0 if n is None else n
        return np.concatenate([self.state(i).reshape(-1, order="F") for i in range(i0, i0 + n)])

    def x(self, i):
        return self._template(self.nx[i]).x

    def make(self, params, group_cells=0, chunk=256):
        """A Batch with grid, boundaries and the initial state uploaded (in
        chunks of instances) and the initial ghost fill done."""
        b = Batch(params, 2, 2, self.nx, group_cells=group_cells)
        b.set_grid(self.x_concat())
        b.set_boundaries(self.typeB())
        for i0 in range(0, self.ninst, chunk):
            n = min(chunk, self.ninst - i0)
            b.upload(self.w_concat(i0, n), i0, n)
        b.getboundary()
        return b


__all__ = ["Batch", "OTBatch", "ot_sizes", "ot_betas", "ot_params", "OT_SIZES"]
