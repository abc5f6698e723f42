"""Shared helpers of the test-suite: drive a Problem through a C-ABI context."""
import numpy as np

from sac_b200 import abi


def start(ctx_cls, P, **kw):
    c = ctx_cls(P.params, **kw) if kw else ctx_cls(P.params)
    c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    c.set_boundaries(P.typeB_packed, P.nB)
    c.upload(P.w)
    c.getboundary(0.0)
    return c


def run(c, nsteps, t0=0.0, it0=0, dts=None, idim=None):
    """Advance nsteps; returns the dt sequence used.  dts forces the steps."""
    t, used = t0, []
    for k in range(nsteps):
        dt = c.getdt(it0 + k) if dts is None else dts[k]
        if idim is None:
            c.advect(dt, t, it0 + k)
        else:
            for d in idim:
                c.advect(dt, t, it0 + k, idimmin=d, idimmax=d)
        used.append(dt)
        t += dt
    return used


def mesh(P, w):
    sl = tuple(slice(2, 2 + n) for n in P.nx)
    return w[sl]


def rel_l2(a, b):
    """Per-variable relative L2 error of a against b (last axis = variable)."""
    out = []
    for iw in range(b.shape[-1]):
        num = np.linalg.norm((a[..., iw] - b[..., iw]).ravel())
        den = np.linalg.norm(b[..., iw].ravel())
        out.append(num / den if den > 0 else num)
    return np.array(out)


def gpu_ctx(params):
    return abi.Context(params)
