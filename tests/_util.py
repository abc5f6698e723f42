"""Shared helpers of the test-suite: drive a Problem through a C-ABI context."""
import numpy as np

from sac_b200 import abi


def start(ctx_cls, P, **kw):
    c = ctx_cls(P.params, **kw) if kw else ctx_cls(P.params)
    c.set_grid(P.ndim, P.ndir, P.ixGhi, P.ixM, P.x)
    c.set_boundaries(P.typeB_packed, P.nB, regions=getattr(P, "regions", None))
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


def gridsetup1_dx(P):
    """Cell widths as gridsetup1 (src/vacgrid.t:585-629) makes them: the ghost
    coordinates, and one more layer, are extrapolated from the two edge mesh cells,
    (1+n) x(edge) - n x(edge-+1), one dimension after the other over the whole
    extended grid; then dx = (x(+1) - x(-1))/2.  Returns dx[..., d] on the full grid."""
    nd = P.ndim
    G = [n + 4 for n in P.nx]
    qx = np.zeros([g + 2 for g in G] + [nd])
    qx[tuple(slice(1, 1 + g) for g in G)] = P.x

    def at(d, i):
        return tuple(i if e == d else slice(None) for e in range(nd))

    for d in range(nd):
        lo, hi = 3, P.nx[d] + 2  # the first and last mesh cell in extended coordinates
        for ix in range(hi + 1, G[d] + 2):
            n = ix - hi
            qx[at(d, ix)] = float(1 + n) * qx[at(d, hi)] - float(n) * qx[at(d, hi - 1)]
        for ix in range(lo - 1, -1, -1):
            n = lo - ix
            qx[at(d, ix)] = float(1 + n) * qx[at(d, lo)] - float(n) * qx[at(d, lo + 1)]
    dx = np.zeros(tuple(G) + (nd,))
    for d in range(nd):
        sl = lambda k: tuple(slice(1 + (k if e == d else 0), 1 + (k if e == d else 0) + G[e])  # noqa: E731
                             for e in range(nd))
        dx[..., d] = 0.5 * (qx[sl(1) + (d,)] - qx[sl(-1) + (d,)])
    return dx


def fp32_rounded(P):
    """A copy of P whose advanced (perturbed) variables are rounded to FP32, as
    the FP32 path stores them; the background stays FP64."""
    import copy

    Q = copy.deepcopy(P)
    npv = 2 * P.ndir + 2
    Q.w[..., :npv] = Q.w[..., :npv].astype(np.float32).astype(np.float64)
    return Q


def fp32_twin(P, nsteps, gpu_cls=None):
    """The FP32 path against the scheme's own sensitivity to FP32 rounding.

    Runs the oracle (FP64) from P's initial state for nsteps with its own getdt,
    then the oracle from the FP32-rounded initial state (the twin) and the FP32
    device path from P's state, both on that dt sequence.  Returns the
    per-variable relative L2 errors over the mesh of the advanced variables:
    (FP32 path vs oracle, twin vs oracle)."""
    import copy

    from oracle.oracle import Oracle
    from sac_b200 import params

    npv = 2 * P.ndir + 2
    o = start(Oracle, P)
    dts = run(o, nsteps)
    wo = mesh(P, o.download())[..., :npv]
    o.close()
    ot = start(Oracle, fp32_rounded(P))
    run(ot, nsteps, dts=dts)
    etw = rel_l2(mesh(P, ot.download())[..., :npv], wo)
    ot.close()
    P32 = copy.deepcopy(P)
    P32.params.precision = params.PREC_FP32
    g = start(gpu_cls or abi.Context, P32)
    run(g, nsteps, dts=dts)
    w32 = mesh(P, g.download())[..., :npv]
    g.close()
    assert np.isfinite(w32).all()
    return rel_l2(w32, wo), etw
