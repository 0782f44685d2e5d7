"""FP64 NumPy restatement of xSPDE 4.21's ensemble-integration path.

TEST INFRASTRUCTURE ONLY.  This module is the CPU oracle that checks the CUDA
path of ``xspde_matlab_b200``.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` may import it; the product never does.

Every function restates one MATLAB function of the reference, cited by
``file:line`` (paths relative to the reference project root).  Arrays keep
MATLAB's shapes -- ``[fields, space..., ens]`` -- and every MATLAB ``reshape`` is
done in column-major order (``order='F'``).  User functions (``deriv``,
``initial``, ``observe``, ``linear``, ``compare``, ``output``) are Python
callables taking the same arguments as their MATLAB counterparts; grid arrays
(``p.x``, ``p.kx`` ...) carry explicit singleton dimensions so that NumPy
broadcasting matches MATLAB's leading-dimension broadcasting.

Noise: the reference draws from MATLAB's Threefry stream.  Here
``p.noisegen``/``p.randomgen`` (the reference's own hooks,
Simulator/xpreferences.m:120-121) default to the counter-based Philox mapping
of ``oracle/philox.py``, which the CUDA path uses too.
"""
import math
import time

import numpy as np

from . import philox


class Struct(dict):
    """MATLAB-struct-like dict with attribute access (p.x == p['x'])."""

    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError as exc:
            raise AttributeError(k) from exc

    def __setattr__(self, k, v):
        self[k] = v

    def copy(self):
        return Struct(self)


def msize(a):
    """MATLAB ``size``: trailing singleton dimensions dropped, at least 2."""
    sz = list(np.shape(a))
    while len(sz) > 2 and sz[-1] == 1:
        sz.pop()
    while len(sz) < 2:
        sz.append(1)
    return sz


def freshape(a, shape):
    return np.reshape(a, shape, order="F")


def fit(a, shape):
    """``reshape(x, shape)`` when the element counts agree, else broadcast."""
    a = np.asarray(a)
    n = int(np.prod(shape))
    if a.size == n:
        return freshape(a, shape)
    if a.ndim < len(shape):
        a = a.reshape(a.shape + (1,) * (len(shape) - a.ndim))
    return np.broadcast_to(a, shape).copy()


def _pad(v, n, fill):
    v = list(np.atleast_1d(v)) if v is not None else []
    if not v:
        v = [fill]
    while len(v) < n:
        v.append(v[-1] if fill is None else fill)
    return v


# ---------------------------------------------------------------------------
# Defaults and grids: Simulator/xpreferences.m, Applications/SPDE/spdpreferences.m,
# Applications/SPDE/xgrid.m
# ---------------------------------------------------------------------------

def _method_name(m):
    if callable(m):
        return m.__name__
    return {"xRK4": "RK4", "xMP": "MP", "xEuler": "Euler", "xRK2": "RK2"}.get(m, m)


def xpreferences(inputs):
    """Fill defaults and derived constants (Simulator/xpreferences.m:11-414)."""
    if isinstance(inputs, dict):
        inputs = [inputs]
    out = []
    origin = 0.0
    for s, pin in enumerate(inputs):
        p = Struct(pin)
        # xSPDE-3 spellings accepted by the reference's users: da/step.
        if "da" in p and "deriv" not in p:
            p.deriv = p.da
        if "step" in p and "method" not in p:
            p.method = p.step
        ens = [int(x) for x in _pad(p.get("ensembles", 1), 3, 1)]      # :26
        p.ensembles = ens
        p.tol = p.get("tol", 1e-20)                                      # :27
        p.dimensions = int(p.get("dimensions", 1))                       # :42
        nd = max(1, p.dimensions)                                        # :43
        p.fields = int(p.get("fields", 1))                               # :44
        if p.dimensions == 0:
            p.points = _pad(p.get("points", [1]), 1, None)
            p.checks = [0]
        else:
            dflt = [51] + [35] * (nd - 1)                                # :56
            pts = list(np.atleast_1d(p.get("points", dflt)))
            p.points = [int(x) for x in pts] + dflt[len(pts):]
            chk = list(np.atleast_1d(p.get("checks", [1] + [0] * (nd - 1))))
            p.checks = [int(x) for x in chk] + [0] * (nd - len(chk))     # :57
        if s > 0:
            p.checks = out[0].checks                                     # :32
        p.iterations = int(p.get("iterations", 4))                       # :59
        p.rawdata = int(p.get("rawdata", 0))                             # :85
        p.auxfields = int(np.atleast_1d(p.get("auxfields", 0))[0])       # :46 (one auxiliary cell)
        p.define = p.get("define", None)                                 # :93
        if "deriv" not in p:
            p.deriv = lambda a, w, p: 0 * a                              # :64
        nz = p.get("noises", None)
        kz = p.get("knoises", None)
        p.knoises = int(np.atleast_1d(kz)[0]) if kz is not None else 0     # :67
        p.noises = (int(np.atleast_1d(nz)[0]) if nz is not None
                    else (0 if kz is not None else p.fields))            # :65-70
        krz = p.get("krandoms", None)
        p.krandoms = int(np.atleast_1d(krz)[0]) if krz is not None else 0  # :73
        p.nfilter = p.get("nfilter", lambda w, p: w)                     # :122, :419-421
        p.rfilter = p.get("rfilter", lambda w, p: w)                     # :123, :423-425
        rz = p.get("inrandoms", None)
        p.inrandoms = (int(np.atleast_1d(rz)[0]) if rz is not None
                       else (0 if krz is not None else p.noises))        # :71-76
        p.ranges = [float(x) for x in _pad(p.get("ranges", [10.0] * nd), nd, 10.0)]  # :81
        st = list(np.atleast_1d(p.get("steps", [1])))
        p.steps = [int(x) for x in st] + [1] * (nd - len(st))            # :82
        org = [origin] + [-r / 2 for r in p.ranges[1:]]                  # :83
        og = list(np.atleast_1d(p.get("origins", org)))
        p.origins = [float(x) for x in og] + org[len(og):]
        p.linear = p.get("linear", None)                                 # :86
        p.seed = int(p.get("seed", 0))                                   # :88
        p.initial = p.get("initial", lambda v, p: 0.0)                   # :92
        p.transfer = p.get("transfer", lambda a, v, p: a)                # :94
        if "method" not in p:                                            # :101-105
            p.method = "RK4" if int(np.prod(ens)) == 1 else "MP"
        p.method = _method_name(p.method)
        p.relerr = p.get("relerr", 1)
        p.propfactor = xpropfactor
        p.prop = xprop
        p.path = p.get("path", xpath)
        p.noisegen = p.get("noisegen", philox_noisegen)                  # :120
        p.randomgen = p.get("randomgen", philox_randomgen)               # :121
        p.nfields = 1
        # cell parameters (:133-160) for the single field cell
        points = list(p.points)
        for d in range(1, nd):
            points[d] = 1 + (points[d] - 1) * p.steps[d]                 # :137
        p.points = points
        dx = [p.ranges[d] / max(1, points[d] - 1) for d in range(nd)]    # :138
        dx = [1.0 if points[d] == 1 else dx[d] for d in range(nd)]       # :139
        p.dx = dx
        p.dv = float(np.prod(dx[1:])) if nd > 1 else 1.0                 # :140
        p.noisefactor = 1.0 / p.dv                                       # :141
        p.knoisefactor = float(np.prod(points[1:])) / p.dv               # :142
        space = points[1:]
        p.space = space
        p.nspace = int(np.prod(space)) if space else 1
        p.ca = [p.fields] + space + [ens[0]]                              # :145
        p.cax = [p.auxfields] + space + [ens[0]]                          # auxiliary cell
        p.dk = [2 * math.pi / (points[d] * dx[d]) for d in range(nd)]    # :165
        p.dk[0] /= p.steps[0]                                            # :166
        p.kfact = [x / math.sqrt(2 * math.pi) for x in dx]               # :167
        p.dt = p.ranges[0] / max(1, points[0] - 1)                       # :174
        p.nscale = p.steps[0] * (1 + p.checks[0]) / p.dt                 # :175
        p.nchk = 1 + int(sum(p.checks))                                  # :182
        p.fbsw = 0
        p.dw = 2 * math.pi / (p.ranges[0] + p.dt)                        # :199
        p.fsc = math.sqrt(2 * math.pi) / p.dw                            # :200
        p0 = np.arange(points[0])
        p.xc = [p.origins[0] + p.dx[0] * p0]                              # :206
        p.kc = [(p0 - points[0] // 2) * p.dw]                             # :203,:207
        p.setboundaries = 0
        if nd > 1:
            _spdpreferences(p)
            _xgrid0(p)
        p.dtr = 0.0
        p.t = p.origins[0]
        if p.method in ("Euler", "Implicit", "RK2"):                     # :213-218
            p.ipsteps = int(p.get("ipsteps", 1))
        else:
            p.ipsteps = int(p.get("ipsteps", 2))
        p.order = int(p.get("order", 0))                                 # :219
        # observables (:224-343)
        obs = p.get("observe", None)
        if obs is None:
            obs = [_xobserve]
        elif callable(obs):
            obs = [obs]
        p.observe = list(obs)
        p.averages = list(range(len(p.observe)))
        tr = p.get("transforms", None)
        if tr is None:
            tr = [[0] * (nd + 1)] * len(p.observe)
        elif not isinstance(tr, (list, tuple)) or not isinstance(tr[0], (list, tuple, np.ndarray)):
            tr = [tr] if not isinstance(tr, (list, tuple)) else list(tr)
        tr = [list(np.atleast_1d(x)) + [0] * (nd + 1) for x in tr]
        while len(tr) < len(p.observe):
            tr.append([0] * (nd + 1))
        p.transforms = [x[: nd + 1] for x in tr]
        p.xk = []
        for n in range(len(p.observe)):
            xk = []
            for j in range(nd):
                if not p.transforms[n][j]:
                    xk.append(p.origins[j] + np.arange(points[j]) * p.dx[j])
                else:
                    start = -points[j] / 2
                    xk.append((start + np.arange(points[j])) * p.dk[j])
            p.xk.append(xk)
        p.d_obs, p.d_av = [], []
        a0 = np.zeros(p.ca, dtype=complex)
        x0 = np.zeros(p.cax, dtype=complex) if p.auxfields else None
        for n in range(len(p.observe)):
            p.nobserve = n
            O = _observe(a0, x0, n, p)
            sz = msize(O)
            if sz[-1] > ens[0] and sz[-1] % ens[0] == 0:                 # :269-272
                szl = sz[-1]
                sz[-1] = szl // ens[0]
                sz.append(ens[0])
            if p.dimensions <= 1:
                lines = int(np.prod(sz[:-1]))
                spaceobs = []
            else:
                lines = sz[0]
                if int(np.prod(sz[1:-1])) == p.nspace:
                    spaceobs = list(space)
                else:
                    spaceobs = sz[1:-1]
            ens1 = sz[-1]
            p.d_obs.append([lines, 1, int(np.prod(spaceobs)) if spaceobs else 1, ens1])
            p.d_av.append([lines, points[0]] + list(spaceobs))
        outs = p.get("output", None)
        if outs is None:
            outs = [None] * len(p.observe)
        elif callable(outs):
            outs = [outs]
        outs = list(outs) + [None] * (len(p.observe) - len(outs))
        p.output = [o if o is not None else (lambda o, p, n=n: o[n]) for n, o in enumerate(outs)]
        p.outputs = list(range(len(p.output)))
        cmp = p.get("compare", None)
        if cmp is None:
            cmp = []
        elif callable(cmp):
            cmp = [cmp]
        p.compare = list(cmp) + [None] * (len(p.output) - len(cmp))
        cut = p.get("cutoff", -1e20)
        p.cutoffs = list(p.get("cutoffs", [])) + [cut] * len(p.output)
        O = [np.zeros(x) for x in p.d_av]
        p.gpoints, p.d_data = [], []
        for n in p.outputs:
            if n >= len(p.xk):
                p.xk.append(p.xk[-1])
                p.transforms.append([0] * (nd + 1))
            g = msize(p.output[n](O, p))
            p.d_data.append(int(np.prod(g)))
            p.gpoints.append(g + [max(3, 1 + p.nchk + p.fbsw)])          # :378-380
            p.xk[n] = list(p.xk[n])
            p.xk[n][0] = p.xc[0]
        ax = p.get("axes", None)
        ax = list(ax) if ax is not None else []
        ax = ax + [None] * (len(p.outputs) - len(ax))
        p.axes = [list(a) + [0] * (nd + 10 - len(a)) if a is not None else [0] * (nd + 10) for a in ax]
        p.ftransforms = p.get("ftransforms", p.transforms)
        out.append(p)
        origin = p.origins[0] + p.ranges[0]                              # :197
    return out


def _xobserve(a, *rest):
    """Default observe: all field components as lines (xpreferences.m:427-446); it
    takes the field and ignores the other cells and p (varargin)."""
    return a


def _spdpreferences(p):
    """k grids and boundary flags (Applications/SPDE/spdpreferences.m:1-73)."""
    nd = p.dimensions
    pts = p.points
    bnd = p.get("boundaries", None)
    bnd = list(bnd) if bnd is not None else []
    # boundaries{c,d} for c = 1: a list indexed by dimension (0-based, d >= 1)
    b = []
    for d in range(nd):
        bd = bnd[d] if d < len(bnd) and bnd[d] is not None else None
        bd = np.zeros((p.fields, 2), dtype=int) if bd is None else np.atleast_2d(np.asarray(bd, dtype=int))
        b.append(bd)
    p.boundaries = b
    p.dkp = [math.pi / ((pts[d] - 1) * p.dx[d]) if pts[d] > 1 else 0.0 for d in range(nd)]  # :16
    p.points2 = [x // 2 for x in pts]
    p.setboundaries = 0
    p.setboundcell = 0
    p.kcp = [[None] * nd for _ in range(p.fields)]
    p.xc = list(p.xc) + [None] * (nd - 1)
    p.kc = list(p.kc) + [None] * (nd - 1)
    p.boundval = [None] * nd
    zero = np.zeros([p.fields] + list(pts[1:]) + [p.ensembles[0]])
    for d in range(1, nd):
        p.boundval[d] = _xboundfun(zero, 0, d, p)                     # :40-43
    for d in range(1, nd):
        n = pts[d]
        p0 = np.arange(n)
        p1 = np.arange(1, n)
        p.xc[d] = p.origins[d] + p0 * p.dx[d]                           # :35
        p.kc[d] = (p0 - p.points2[d]) * p.dk[d]                         # :36
        if np.any(b[d] != 0):
            p.setboundaries = 1
            p.setboundcell = 1
        typ = b[d][:, 0] + 2 * b[d][:, 1]
        for j in range(p.fields):
            t = int(typ[j])
            if t == -3:
                k = p0 * p.dkp[d]
            elif t == -1:
                k = np.concatenate([[0.0], p1 - 0.5]) * p.dkp[d]
            elif t == 0:
                k = np.fft.ifftshift(p.kc[d])
            elif t == 1:
                k = np.concatenate([p1 - 0.5, [0.0]]) * p.dkp[d]
            elif t == 3:
                k = p0 * p.dkp[d]
            else:
                raise ValueError("Invalid boundary type: %r" % (b[d][j],))
            p.kcp[j][d] = k
    p.boundfun = p.get("boundfun", _xboundfun)


def _xboundfun(ac, c, d, p):
    """Default boundary values: zeros (spdpreferences.m:75-96)."""
    sz = list(np.shape(ac))
    s1 = sz[0]
    sz[0] = 1
    sz[d] = 1
    return [[np.zeros(sz), np.zeros(sz)] for _ in range(s1)]


def _bshape(nd, d, n):
    """Shape with n in MATLAB dimension d (0-based numpy axis d) for a field array."""
    sh = [1] * (nd + 1)
    sh[d] = n
    return sh


def _xgrid0(p):
    """Lattice and k-space grids in propagation order (xgrid.m:17-48)."""
    nd = p.dimensions
    pts = p.points
    p.r = [None] * max(4, nd)
    p.k = [None] * max(4, nd)
    for d in range(1, nd):
        p.r[d] = p.xc[d].reshape(_bshape(nd, d, pts[d]))
        if not np.any(p.boundaries[d] != 0):
            p.k[d] = p.kcp[0][d].reshape(_bshape(nd, d, pts[d]))
        else:
            kk = np.stack([p.kcp[j][d] for j in range(p.fields)])
            sh = _bshape(nd, d, pts[d])
            sh[0] = p.fields
            p.k[d] = kk.reshape(sh)
    p.x, p.y, p.z = p.r[1], p.r[2], p.r[3]
    p.kx, p.ky, p.kz = p.k[1], p.k[2], p.k[3]


def xgrid_out(n, p):
    """Output-grid coordinate arrays for compare functions (xgrid.m:49-56)."""
    q = p.copy()
    xk = p.xk[n]
    d = len(xk)
    r = []
    for j in range(d):
        sh = [1] * (d + 1)
        sh[j + 1] = len(xk[j])
        r.append(np.asarray(xk[j], dtype=float).reshape(sh))
    r += [None] * (4 - len(r))
    q.r = r
    q.t, q.x, q.y, q.z = r[0], r[1], r[2], r[3]
    q.w, q.kx, q.ky, q.kz = r[0], r[1], r[2], r[3]
    q.rr = r
    return q


# ---------------------------------------------------------------------------
# Interaction-picture operators: Applications/SPDE/xpropfactor.m, xprop.m,
# xtransform.m, xdst1-3.m, xdct1-3.m, xpatch.m, xsetbound.m
# ---------------------------------------------------------------------------

def xpropfactor(p):
    """propagator = exp(L dt), dt = dtr/ipsteps (xpropfactor.m:26-58)."""
    dt = p.dtr / p.ipsteps                                               # :28
    nd = p.dimensions
    if nd > 1:
        p.D = [None] + [1j * p.k[d] if p.k[d] is not None else None for d in range(1, max(4, nd))]
        p.Dx, p.Dy, p.Dz = p.D[1], p.D[2], p.D[3]
    da = [0.0] * nd
    if p.linear is None or (not callable(p.linear) and p.linear == 0):
        return 1, da
    L = np.asarray(p.linear(p), dtype=complex)
    prop = np.exp(L * dt)                                                # :39
    if nd > 1 and p.setboundaries:
        fda = dt / math.pi ** 2                                          # :45
        for d in range(1, nd):
            Lf = np.broadcast_to(L, [max(L.shape[0], 1)] + p.space + [1]) if L.ndim else L
            idx1 = [slice(None)] + [0] * (nd - 1) + [0]
            idx2 = list(idx1)
            idx2[d] = 1
            L1 = Lf[tuple(idx1)]
            L2 = Lf[tuple(idx2)]
            da[d] = -(L2 - L1) * fda * p.ranges[d] ** 2                   # :50
    return prop, da


def _swap(a, ax):
    return np.moveaxis(a, ax, -1)


def xdct1(a, ax):
    """DCT-I via a 2(N-1)-point FFT, real and imaginary parts apart (xdct1.m:8-20)."""
    if np.iscomplexobj(a) and np.any(np.imag(a) != 0):
        return xdct1(np.real(a), ax) + 1j * xdct1(np.imag(a), ax)
    a = np.real(a)
    x = _swap(a, ax)
    N = x.shape[-1]
    ext = np.concatenate([x, np.flip(x[..., 1:N - 1], -1)], axis=-1)
    y = np.fft.fft(ext, axis=-1)[..., :N] * math.sqrt(1.0 / (2 * (N - 1)))
    return np.moveaxis(y, -1, ax)


def xdst1(a, ax):
    """DST-I on the interior points, end points zeroed (xdst1.m:8-19)."""
    x = _swap(np.asarray(a, dtype=complex), ax)
    N = x.shape[-1]
    n2 = 2 * (N - 1)
    ext = np.zeros(x.shape[:-1] + (n2,), dtype=complex)
    ext[..., 1:N - 1] = x[..., 1:N - 1]
    ext[..., N:n2] = -np.flip(x[..., 1:N - 1], -1)
    y = np.fft.fft(ext, axis=-1)
    out = x.copy()
    out[..., 1:N - 1] = y[..., 1:N - 1] * math.sqrt(2.0 / (N - 1)) / (-2j)
    out[..., 0] = 0
    out[..., N - 1] = 0
    return np.moveaxis(out, -1, ax)


def xdct2(a, ax):
    """DCT-II on the first N-1 points (xdct2.m:11-29)."""
    if np.iscomplexobj(a):
        return xdct2(np.real(a), ax) + 1j * xdct2(np.imag(a), ax)
    x = _swap(a, ax)
    N = x.shape[-1]
    M = N - 1
    ext = np.zeros(x.shape[:-1] + (2 * M,))
    ext[..., :M] = x[..., :N - 1]
    y = np.fft.fft(ext, axis=-1)
    post = np.exp(-1j * math.pi / (2 * M) * np.arange(M))
    ct = np.zeros(x.shape)
    ct[..., :N - 1] = np.real(y[..., :M] * post)
    ct = ct * math.sqrt(2.0 / M)
    return np.moveaxis(ct, -1, ax)


def xdct3(a, ax):
    """DCT-III on the first N-1 points (xdct3.m:13-33)."""
    if np.iscomplexobj(a):
        return xdct3(np.real(a), ax) + 1j * xdct3(np.imag(a), ax)
    x = _swap(a, ax)
    N = x.shape[-1]
    M = N - 1
    ext = np.zeros(x.shape[:-1] + (2 * M,), dtype=complex)
    ext[..., :M] = x[..., :N - 1]
    ext[..., 0] = 0
    pre = np.exp(-1j * math.pi / (2 * M) * np.arange(M))
    ext[..., :M] = ext[..., :M] * pre
    y = np.fft.fft(ext, axis=-1)
    ct = np.zeros(x.shape)
    ct[..., :N - 1] = np.real(y[..., :M])
    ct[..., :N - 1] = ct[..., :N - 1] + 0.5 * x[..., :1]
    ct = ct * math.sqrt(2.0 / M)
    return np.moveaxis(ct, -1, ax)


def xdst2(a, ax):
    """DST-II on the last N-1 points (xdst2.m:13-33)."""
    if np.iscomplexobj(a):
        return xdst2(np.real(a), ax) + 1j * xdst2(np.imag(a), ax)
    x = _swap(a, ax)
    N = x.shape[-1]
    M = N - 1
    ext = np.zeros(x.shape[:-1] + (2 * M,), dtype=complex)
    ext[..., :M] = x[..., 1:N]
    pre = np.exp(-1j * math.pi / M * np.arange(M))
    post = np.exp(-1j * math.pi / (2 * M) * np.arange(1, M + 1))
    ext[..., :M] = ext[..., :M] * pre
    y = np.fft.fft(ext, axis=-1)
    ct = np.zeros(x.shape)
    ct[..., 1:N] = -np.imag(y[..., :M] * post)
    ct = ct * math.sqrt(2.0 / M)
    return np.moveaxis(ct, -1, ax)


def xdst3(a, ax):
    """DST-III on the last N-1 points (xdst3.m:12-35)."""
    if np.iscomplexobj(a):
        return xdst3(np.real(a), ax) + 1j * xdst3(np.imag(a), ax)
    x = _swap(a, ax)
    N = x.shape[-1]
    M = N - 1
    ext = np.zeros(x.shape[:-1] + (2 * M,), dtype=complex)
    ext[..., :M] = x[..., 1:N]
    ext[..., M - 1] = 0
    pre = np.exp(-1j * math.pi / (2 * M) * np.arange(M))
    post = np.exp(-1j * math.pi / M * (np.arange(M) + 0.5))
    ext[..., :M] = ext[..., :M] * pre
    y = np.fft.fft(ext, axis=-1)
    ct = np.zeros(x.shape)
    ct[..., 1:N] = -np.imag(y[..., :M] * post)
    alt = np.cumprod(-np.ones(M))
    ct[..., 1:N] = ct[..., 1:N] - 0.5 * (alt * x[..., N - 1:N])
    ct = ct * math.sqrt(2.0 / M)
    return np.moveaxis(ct, -1, ax)


_FWD = {-3: xdct1, -1: xdst3, 1: xdct3, 3: xdst1}
_INV = {-3: xdct1, -1: xdst2, 1: xdct2, 3: xdst1}


def xtransform(a, inv, p):
    """Per-component spectral transform over every space dimension (xtransform.m:21-70)."""
    nd = p.dimensions
    a = np.array(a, dtype=complex)
    for i in range(a.shape[0]):
        at = a[i:i + 1]
        for d in range(1, nd):
            if a.shape[d] > 1:
                b = p.boundaries[d]
                t = int(b[i, 0] + 2 * b[i, 1])
                if t == 0:
                    at = np.fft.ifft(at, axis=d) if inv else np.fft.fft(at, axis=d)
                else:
                    at = (_INV if inv else _FWD)[t](at, d)
        a[i:i + 1] = at
    return a


def xpatch(ac, p):
    """Boundary patch for non-periodic transforms (xpatch.m:24-62)."""
    a = ac
    pa = 0.0
    lp = 0.0
    nd = p.dimensions
    sx = a.shape
    for d in range(1, nd):
        bnd = p.boundaries[d]
        typ = bnd[:, 0] + 2 * bnd[:, 1]
        if np.any(typ) and sx[d] > 1:
            pa = np.zeros(sx, dtype=complex)
            lp = np.zeros(sx, dtype=complex)
            b = p.boundfun(ac, 0, d, p)
            xa = p.origins[d]
            dx = p.ranges[d]
            x = p.r[d] - xa
            for i in range(sx[0]):
                t = int(typ[i])
                sl = (slice(i, i + 1),)
                if t == -3:
                    db = (b[i][1] - b[i][0]) / dx
                    pa[sl] = pa[sl] + b[i][0] * x + 0.5 * x ** 2 * db
                    dai = np.asarray(p.da[d]).reshape(-1)
                    lp[sl] = lp[sl] + db * dai[min(i, dai.size - 1)]
                elif t == -1:
                    pa[sl] = pa[sl] + b[i][0] + x * b[i][1]
                elif t == 0:
                    pass
                elif t == 1:
                    pa[sl] = pa[sl] + b[i][1] + (x - dx) * b[i][0]
                elif t == 3:
                    db = (b[i][1] - b[i][0]) / dx
                    pa[sl] = pa[sl] + b[i][0] + x * db
                else:
                    raise ValueError("Invalid boundary")
    return a - pa, pa, 0, lp


def xsetbound(ac, p):
    """Impose Dirichlet boundary values (xsetbound.m:30-63)."""
    a = np.array(ac, dtype=complex)
    nd = p.dimensions
    bval = [None] * nd
    sz = a.shape
    if int(np.prod(sz[1:nd])) > 1:
        for d in range(1, nd):
            bound = p.boundaries[d]
            if np.any(bound != 0):
                bval[d] = p.boundfun(a, 0, d, p)
                if np.any(bound == 1):
                    bv = bval[d]
                    for i in range(sz[0]):
                        if bound[i, 0] == 1:
                            idx = [slice(i, i + 1)] + [slice(None)] * (a.ndim - 1)
                            idx[d] = slice(0, 1)
                            a[tuple(idx)] = bv[i][0]
                        if bound[i, 1] == 1:
                            idx = [slice(i, i + 1)] + [slice(None)] * (a.ndim - 1)
                            idx[d] = slice(sz[d] - 1, sz[d])
                            a[tuple(idx)] = bv[i][1]
    return a, bval


def xprop(a, p):
    """One interaction-picture propagation a <- T^-1[P . T a] (xprop.m:17-46)."""
    bv = 0
    if not (np.isscalar(p.propagator) and p.propagator == 1):
        pat = 0.0
        if p.setboundcell:
            a, pat, sw, patlp = xpatch(a, p)
            pat = pat + patlp
        at = xtransform(a, 0, p)
        at = p.propagator * at
        a = xtransform(at, 1, p) + pat
    if p.setboundaries:
        a, bv = xsetbound(a, p)
    return a, bv


# ---------------------------------------------------------------------------
# Steppers: Applications/SDE/MP.m, RK4.m, Euler.m, RK2.m, Implicit.m
# ---------------------------------------------------------------------------

class Cells(list):
    """Several noise or random cells (Gaussian, then k-filtered), passed to the
    user's functions as separate arguments: p.deriv{c}(a{:}, xi{:}, p) (MP.m:16),
    p.initial(v{:}, p) (xensemble.m:60)."""


def call_cells(fn, first, cells, p):
    if isinstance(cells, Cells):
        return fn(*([] if first is None else [first]), *cells, p)
    return fn(*([] if first is None else [first]), cells, p)


def _deriv(a, w, p):
    return fit(call_cells(p.deriv, a, w, p), p.ca)


def MP(a, xi, p):
    """Midpoint IP step (Applications/SDE/MP.m:10-27)."""
    q = p.copy()
    dt = q.dtr / 2.0                                                     # :10
    a, q.boundval = q.prop(a, q)                                         # :11
    q.t = q.t + dt                                                       # :12
    a0 = a
    for _ in range(q.iterations):                                        # :14
        a = a0 + _deriv(a, xi, q) * dt                                   # :16
        if q.setboundaries:
            a, q.boundval = xsetbound(a, q)                              # :18-20
    a = 2 * a - a0                                                       # :23
    q.t = q.t + dt                                                       # :25
    a, _ = q.prop(a, q)                                                  # :26
    return a


def RK4(a, xi, p):
    """Fourth-order Runge-Kutta IP step, one noise for all stages (RK4.m:7-42)."""
    q = p.copy()
    dt = 0.5 * q.dtr
    if q.setboundaries:
        a, q.boundval = xsetbound(a, q)
    a1 = a + _deriv(a, xi, q) * dt
    a1, q.boundval = q.prop(a1, q)
    a, _ = q.prop(a, q)
    q.t = q.t + dt
    a2 = a + _deriv(a1, xi, q) * dt
    if q.setboundaries:
        a2, q.boundval = xsetbound(a2, q)
    a3 = a + _deriv(a2, xi, q) * 2 * dt
    if q.setboundaries:
        a3, _ = xsetbound(a3, q)
    a = (a1 + 2 * a2 + a3 - a) / 3
    q.t = q.t + dt
    a, _ = q.prop(a, q)
    a3, q.boundval = q.prop(a3, q)
    a = a + _deriv(a3, xi, q) * dt / 3
    if q.setboundaries:
        a, _ = xsetbound(a, q)
    return a


def Euler(a, xi, p):
    """Euler IP step (Euler.m:6-10)."""
    a = a + _deriv(a, xi, p) * p.dtr
    a, _ = p.prop(a, p)
    return a


def RK2(ac, xi, p):
    """Second-order Runge-Kutta IP step (RK2.m:7-25)."""
    q = p.copy()
    dt = q.dtr
    a = ac + _deriv(ac, xi, q) * dt
    q.t = q.t + dt
    ac, _ = q.prop(ac, q)
    if q.setboundaries:
        ac, q.boundval = xsetbound(ac, q)
    a, _ = q.prop(a, q)
    if q.setboundaries:
        a, q.boundval = xsetbound(a, q)
    ac = ac + _deriv(a, xi, q) * dt
    ac = (a + ac) / 2
    return ac


def Implicit(a, xi, p):
    """Implicit (iterated Euler) IP step (Implicit.m:8-17)."""
    q = p.copy()
    dt = q.dtr
    q.t = q.t + dt
    a0 = a
    for _ in range(q.iterations):
        a = a0 + _deriv(a, xi, q) * dt
    a, _ = q.prop(a, q)
    return a


METHODS = {"MP": MP, "RK4": RK4, "Euler": Euler, "RK2": RK2, "Implicit": Implicit}


# ---------------------------------------------------------------------------
# Noise hooks: Simulator/xnoise.m, Simulator/xrandom.m (Philox stream)
# ---------------------------------------------------------------------------

def _kcells(nk, draw, filt, scale, p):
    """k-filtered cell (xnoise.m:40-46, xrandom.m:24-29): real normals on the
    k-space lattice from the k stream, the filter, xift (ifft along each space
    dimension, Applications/SPDE/xift.m), times the scale."""
    z = philox.normals(nk, p.nspace, p.ensembles[0], draw, p.block, p.seed, p.get("seq", 0), kstream=True)
    zk = freshape(z, [nk] + p.space + [p.ensembles[0]]).astype(complex)
    zk = np.asarray(filt(zk, p), dtype=complex)                          # :42
    for d in range(1, p.dimensions):                                     # xift.m:8-10
        zk = np.fft.ifft(zk, axis=d)
    return zk * scale                                                    # :43


def philox_noisegen(w1, nc, s, p):
    """p.noisegen replacement: Gaussian noise * sqrt(s*noisefactor), coarse
    pass averages two fine draws (xnoise.m:29-38).  The draw index comes
    from ``p.draw`` which xpath advances once per call.  With knoises the
    cells [Gaussian (if noises > 0), k-filtered] come as ``Cells``."""
    if p.knoises > 0:
        cells = Cells()
        if p.noises > 0:
            z = philox.normals(p.noises, p.nspace, p.ensembles[0], p.draw, p.block, p.seed, p.get("seq", 0),
                               p.space[0] if p.space else 1)
            cells.append(freshape(z, [p.noises] + p.space + [p.ensembles[0]]) * math.sqrt(s * p.noisefactor))
        cells.append(_kcells(p.knoises, p.draw, p.nfilter, math.sqrt(s * p.knoisefactor), p))
        if w1 is not None and p.checks[0] and nc == 2:                   # :33-35, :45-47
            cells = Cells((x + y) / 2 for x, y in zip(cells, w1))
        return cells
    if p.noises <= 0:
        return 0
    z = philox.normals(p.noises, p.nspace, p.ensembles[0], p.draw, p.block, p.seed, p.get("seq", 0),
                       p.space[0] if p.space else 1)
    w = freshape(z, [p.noises] + p.space + [p.ensembles[0]])
    w = w * math.sqrt(s * p.noisefactor)                                 # :32
    if w1 is not None and p.checks[0] and nc == 2:                       # :33-35
        w = (w + w1) / 2
    return w


def philox_randomgen(p):
    """p.randomgen replacement: initial Gaussian randoms * sqrt(noisefactor)
    (xrandom.m:20-23), Philox draw 0; with krandoms the cells [Gaussian (if
    inrandoms > 0), k-filtered * sqrt(knoisefactor)] (xrandom.m:24-29)."""
    if p.krandoms > 0:
        cells = Cells()
        if p.inrandoms > 0:
            z = philox.normals(p.inrandoms, p.nspace, p.ensembles[0], 0, p.block, p.seed, p.get("seq", 0),
                               p.space[0] if p.space else 1)
            cells.append(freshape(z, [p.inrandoms] + p.space + [p.ensembles[0]]) * math.sqrt(p.noisefactor))
        cells.append(_kcells(p.krandoms, 0, p.rfilter, math.sqrt(p.knoisefactor), p))
        return cells
    if p.inrandoms <= 0:
        return 0
    z = philox.normals(p.inrandoms, p.nspace, p.ensembles[0], 0, p.block, p.seed, p.get("seq", 0),
                       p.space[0] if p.space else 1)
    v = freshape(z, [p.inrandoms] + p.space + [p.ensembles[0]])
    return v * math.sqrt(p.noisefactor)


# ---------------------------------------------------------------------------
# Observables: Simulator/xdata.m, Applications/SPDE/Int.m, Ave.m, xnft.m
# ---------------------------------------------------------------------------

def xnft(a, trans, p):
    """Normalised spatial Fourier transform (xnft.m:23-31)."""
    a = np.array(a, dtype=complex)
    for d in range(1, min(p.dimensions, len(trans))):
        if trans[d] > 0 and a.shape[d] > 1:
            a = np.fft.fft(a, axis=d) * p.kfact[d]
    return a


def _transform_obs(a, n, p):
    tr = p.transforms[n]
    if sum(tr[1:p.dimensions]) > 0:
        return xnft(a, tr, p)
    return a


def _observe(a, x, n, p):
    """observe{n}(a{:}, p) on the (transformed) cells: the field, then the
    auxiliary cell when there is one (xdata.m:25-30)."""
    a = _transform_obs(a, n, p)
    if p.auxfields:
        return np.asarray(p.observe[n](a, _transform_obs(x, n, p), p))
    return np.asarray(p.observe[n](a, p))


def xdata(a, n, p, x=None):
    """Ensemble mean of observe{n} at the current time (xdata.m:21-86); x is
    the auxiliary cell (p.auxfields)."""
    p.nobserve = n
    obs = _observe(a, x, n, p)
    obs = fit(obs, p.d_obs[n])
    return np.mean(obs, axis=3)                                          # :84


def Int(o, *args):
    """Space integral with optional bounds (Applications/SPDE/Int.m:23-71)."""
    p = args[-1]
    dx = list(p.dx)
    b = np.zeros((p.dimensions, 2))
    if len(args) >= 2:
        dx = list(np.atleast_1d(args[0]))
    if len(args) >= 3:
        b = np.atleast_2d(np.asarray(args[1], dtype=float))
    o = np.asarray(o)
    sh = [o.shape[0]] + p.space + [p.ensembles[0]]
    o = fit(o, sh)
    maxind = min(o.ndim, len(dx))
    dx[0] = 0.0
    for i in range(maxind):
        d = dx[i]
        if d > 0:
            if i >= b.shape[0] or b[i, 0] >= b[i, 1]:
                o = np.sum(o, axis=i, keepdims=True) * d
            else:
                x = p.xc[i]
                j = int(math.floor((b[i, 0] - x[0]) / d))
                acc = 0
                while j < len(x) and x[j] <= b[i, 1]:
                    acc = acc + np.take(o, [j], axis=i) * d
                    j += 1
                o = acc
    return o


def Ave(o, *args):
    """Lattice average (Applications/SPDE/Ave.m:14-34)."""
    p = args[-1]
    av = args[0] if len(args) == 2 else [1] * p.dimensions
    o = np.asarray(o)
    maxind = min(o.ndim, len(av), p.dimensions)
    for i in range(1, maxind):
        if av[i] > 0:
            o = np.mean(o, axis=i, keepdims=True)
    return o


def D2(a, d, p):
    """Central second difference along dimension d (Applications/SPDE/D2.m:21-77),
    cell 1, all components, propagation use (p.indext = 0)."""
    a = np.asarray(a)
    dx = p.dx[d]
    out = (np.roll(a, -1, axis=d) + np.roll(a, 1, axis=d) - 2 * a) / dx ** 2
    bnd = p.boundaries[d]
    bval = p.boundval[d] if np.any(bnd == -1) else None
    sx = a.shape[d]
    for i in range(a.shape[0]):
        if bnd[i, 0] != 0:
            lo = [slice(i, i + 1)] + [slice(None)] * (a.ndim - 1)
            lo2 = list(lo)
            lo[d] = slice(0, 1)
            lo2[d] = slice(1, 2)
            if bnd[i, 0] == -1:
                out[tuple(lo)] = 2 * ((a[tuple(lo2)] - a[tuple(lo)]) / dx - bval[i][0]) / dx
            else:
                out[tuple(lo)] = out[tuple(lo2)]
            hi = [slice(i, i + 1)] + [slice(None)] * (a.ndim - 1)
            hi2 = list(hi)
            hi[d] = slice(sx - 1, sx)
            hi2[d] = slice(sx - 2, sx - 1)
            if bnd[i, 1] == -1:
                out[tuple(hi)] = 2 * (bval[i][1] + (a[tuple(hi2)] - a[tuple(hi)]) / dx) / dx
            else:
                out[tuple(hi)] = out[tuple(hi2)]
    return out


def D1(a, d, p):
    """Central first difference along dimension d (Applications/SPDE/D1.m:62-105),
    cell 1, propagation use."""
    a = np.asarray(a)
    dx = p.dx[d]
    out = (np.roll(a, -1, axis=d) - np.roll(a, 1, axis=d)) / (2 * dx)
    bnd = p.boundaries[d]
    bval = p.boundval[d] if np.any(bnd == -1) else None
    for i in range(a.shape[0]):
        lo = [slice(i, i + 1)] + [slice(None)] * (a.ndim - 1)
        hi = list(lo)
        lo[d] = slice(0, 1)
        hi[d] = slice(a.shape[d] - 1, a.shape[d])
        if bnd[i, 0] == -1:
            out[tuple(lo)] = bval[i][0]
        if bnd[i, 1] == -1:
            out[tuple(hi)] = bval[i][1]
    return out


# ---------------------------------------------------------------------------
# Path and ensemble drivers: Simulator/xpath.m, Simulator/xensemble.m
# ---------------------------------------------------------------------------

def xpath(a, nc, p):
    """Time loop: noise, method, observe at step 1 (xpath.m:16-107).

    ``p.draw`` counts ``p.noisegen`` calls (the Philox draw index, from 1)."""
    P1 = p.points[0]
    S = p.steps[0]
    av = [np.zeros(x, dtype=complex) for x in p.d_av]
    method = METHODS[p.method]
    w = None
    p.draw = 0
    spectrum = any(tr[0] for tr in p.transforms)                         # xpreferences.m:246
    aft = np.zeros((P1 * S,) + np.shape(a), dtype=complex) if spectrum else None
    # raw{l}: [fields, points(1), space, ens] (xpreferences.m:148)
    raw = np.zeros((np.shape(a)[0], P1) + np.shape(a)[1:], dtype=complex) if p.rawdata else None
    # auxiliary cell (p.auxfields, p.define): set by xensemble at the start of the path
    x = np.array(p.aux0, dtype=complex) if p.auxfields else None
    aftx = np.zeros((P1 * S,) + np.shape(x), dtype=complex) if (spectrum and p.auxfields) else None
    n1 = -1
    for n in range(P1):                                                  # :29
        for step in range(S):                                            # :30
            n1 += 1                                                      # :31
            if n > 0 or step > 0 or P1 == 1:                             # :32
                for checks in range(p.checks[0] + 1):                    # :33
                    p.draw += 1
                    w = p.noisegen(w, nc, p.nscale, p)                   # :34
                    if nc == 1 or checks == 1:                           # :35
                        if p.auxfields:                                  # :36-38
                            x = fit(np.asarray(call_cells(p.define, a, w, p), dtype=complex), p.cax)
                        a = method(a, w, p)                              # :42
                        if p.auxfields:                                  # :42-44 (same p.t, same noise)
                            x = 0.5 * (x + fit(np.asarray(call_cells(p.define, a, w, p), dtype=complex), p.cax))
                        if spectrum:                                     # :46-54
                            if checks == 1 and nc == 1:
                                aft[n1] = (a + aft[n1]) / 2
                                if p.auxfields:
                                    aftx[n1] = (x + aftx[n1]) / 2
                            else:
                                aft[n1] = a
                                if p.auxfields:
                                    aftx[n1] = x
                        w = None                                         # :56
                        p.t = p.t + p.dtr                                # :57
            elif spectrum:                                               # :64-68
                aft[n1] = a
                if p.auxfields:
                    aftx[n1] = x
            if step == 0:                                                # :73
                if p.rawdata:                                            # :73-78
                    raw[:, n] = a
                for o in p.averages:
                    if not p.transforms[o][0]:
                        r = xdata(a, o, p, x)
                        L = p.d_av[o][0]
                        av[o][:, n] = freshape(r, [L] + list(p.d_av[o][2:]))
    if spectrum:                                                         # :90-106
        nt = P1 * S
        f = np.fft.fftshift(np.fft.ifft(aft, axis=0) * p.fsc, axes=0)   # ifft(aft, P1 S, 2) * fsc, fftshift
        fx = np.fft.fftshift(np.fft.ifft(aftx, axis=0) * p.fsc, axes=0) if p.auxfields else None
        sel = np.arange(P1) - P1 // 2 + nt // 2                          # specpts = plotpts + floor(S P1/2) + 1
        for n in range(P1):
            for o in p.averages:
                if p.transforms[o][0]:
                    r = xdata(f[sel[n]], o, p, fx[sel[n]] if p.auxfields else None)
                    L = p.d_av[o][0]
                    av[o][:, n] = freshape(r, [L] + list(p.d_av[o][2:]))
    return a, av, raw


AUX_DRAW = 0xFFFFFFFF  # Philox draw index of the noise for the initial auxiliary cell


def initial_aux(a, nc, p):
    """Initial auxiliary cell (xensemble.m:74-77): p.define(a, w, p) on one
    noise draw of its own (Philox draw AUX_DRAW), at the current p.t; stored
    in p.aux0 for the path."""
    if not p.auxfields:
        return
    p.draw = AUX_DRAW
    w = p.noisegen(None, nc, p.nscale, p)
    p.aux0 = fit(np.asarray(call_cells(p.define, a, w, p), dtype=complex), p.cax)


def xensemble(npar, inputs):
    """Serial ensembles, checks and moments (xensemble.m:12-108).

    Returns ``data[s][o]``: columns 1..m are (extrapolated) fine, coarse
    block means, column m1 the mean of squared fine block means."""
    seq = len(inputs)
    p1 = inputs[0]
    ne = 1.0 / (p1.ensembles[1] * p1.ensembles[2]) - 1                  # :17
    m = p1.fbsw + p1.nchk                                                # :18
    m1 = max(3, m + 1)                                                   # :19
    data = [[np.zeros((inputs[s].d_data[o], m1)) for o in inputs[s].outputs] for s in range(seq)]
    raws = [[[None] * p1.ensembles[1] for _ in range(p1.nchk)] for _ in range(seq)]  # :15
    D = [dict() for _ in range(seq)]
    for j in range(p1.ensembles[1]):                                     # :25
        block = (npar - 1) + j * p1.ensembles[2]                         # :26
        for nc in range(1, p1.nchk + 1):                                 # :27
            b = None
            for s in range(seq):                                         # :36
                p = inputs[s].copy()
                p.block = block
                p.seq = s
                if p.checks[0] and nc != 2:                              # :41-45
                    p.dtr = p.dt / (2 * p.steps[0])
                else:
                    p.dtr = p.dt / p.steps[0]
                p.propagator, p.da = p.propfactor(p)                     # :47
                v = p.randomgen(p)                                       # :53
                p.t = p.origins[0]
                if s == 0:
                    a = call_cells(p.initial, None, v, p)                # :60
                else:
                    a = p.transfer(b, v, p)                              # :62
                a = fit(np.asarray(a, dtype=complex), p.ca)              # :64
                if p.dimensions > 1 and p.setboundcell:                  # :67-72
                    p.t = p.origins[0] - 1
                    for d in range(1, p.dimensions):
                        p.boundval[d] = p.boundfun(a, 0, d, p)
                initial_aux(a, nc, p)                                    # :74-77
                p.t = p.origins[0]
                b, av, r = p.path(a, nc, p)                              # :79
                raws[s][nc - 1][j] = r
                for o in p.outputs:                                      # :84
                    if p.d_data[o] > 0:
                        nes = 1 + ne
                        Dv = np.real(np.asarray(p.output[o](av, p)))
                        D[s][(nc, o)] = freshape(Dv, [-1])               # :88
                        if nc == p.nchk:                                 # :92
                            if p1.checks[0] and p.order > 0:             # :93-97
                                Del = (D[s][(1, o)] - D[s][(2, o)]) / (2 ** p.order - 1.0)
                                D[s][(2, o)] = D[s][(1, o)]
                                D[s][(1, o)] = D[s][(1, o)] + Del
                            for n1 in range(1, m + 1):                   # :98-100
                                data[s][o][:, n1 - 1] += D[s][(n1, o)] * nes
                            data[s][o][:, m1 - 1] += D[s][(1, o)] ** 2 * nes  # :101
    return data, raws


# ---------------------------------------------------------------------------
# Control and error columns: Simulator/xsim.m, Applications/SPDE/xcompress.m
# ---------------------------------------------------------------------------

def xcompress(n, data, p, xk):
    """Reduce output arrays to the requested axes (xcompress.m:18-70)."""
    axes = list(p.axes[n])
    x = list(xk)
    g = p.gpoints[n]
    d = len(g) - 2
    rank = data.ndim
    np_ = list(data.shape) + [1] * d
    mid = [1 + v // 2 for v in np_]
    for ndim in range(d):
        ind = axes[ndim]
        xnd = x[ndim]
        if np.size(xnd) > 1:
            if ndim + 1 <= p.dimensions and ndim < len(p.ftransforms[n]) and p.ftransforms[n][ndim]:
                xnd = p.kc[ndim]
            if np.isscalar(ind) or np.size(ind) == 1:
                ind = int(np.atleast_1d(ind)[0])
                if ind == 0:
                    ind = list(range(1, np_[ndim + 1] + 1))
                elif ind == -1:
                    ind = [mid[ndim + 1]]
                elif ind == -2:
                    ind = [np_[ndim + 1]]
                else:
                    ind = [ind]
            ind = [int(i) for i in np.atleast_1d(ind)]
            if np_[ndim + 1] > len(ind):
                n1 = int(np.prod(np_[: ndim + 1]))
                n2 = np_[ndim + 1]
                n3 = int(np.prod(np_[ndim + 2:]))
                data = freshape(data, [n1, n2, n3])
                np_[ndim + 1] = len(ind)
                data = data[:, [i - 1 for i in ind], :]
            else:
                ind = ind[: np_[ndim + 1]]
            x[ndim] = np.asarray(xnd)[[i - 1 for i in ind]]
        axes[ndim] = list(range(1, np.size(x[ndim]) + 1))
    data = freshape(data, np_[:rank])
    return data, x


def xsim(*inputs):
    """Run ensembles and compute error columns (xsim.m:28-214).

    Returns (error, data, input) like the reference, and raw as a fourth value
    when an input sets p.rawdata: raw[s][nc][k] is the [fields, points(1), space,
    ens(1)] field array of sequence s, check pass nc and ensemble k = j + ens(2) npar
    (xsim.m:42-57)."""
    t0 = time.perf_counter()
    if len(inputs) == 1 and isinstance(inputs[0], (list, tuple)):
        inputs = inputs[0]
    inp = xpreferences(list(inputs))
    p = inp[0]
    seq = len(inp)
    ne = p.ensembles[1] * p.ensembles[2]                                 # :36
    n1 = ne - 1
    nc1 = p.nchk + p.fbsw
    sx = max(3, 1 + nc1)                                                 # :40
    err = np.zeros(6)
    data = None
    raw = [[[None] * (p.ensembles[1] * p.ensembles[2]) for _ in range(p.nchk)] for _ in range(seq)]  # :42
    for npar in range(1, p.ensembles[2] + 1):                            # :50-60
        dp, rp = xensemble(npar, inp)
        data = dp if data is None else [[x + y for x, y in zip(a, b)] for a, b in zip(data, dp)]
        for s in range(seq):                                             # :54, :57 raw(:,:,:,npar)
            for nc in range(p.nchk):
                for j in range(p.ensembles[1]):
                    raw[s][nc][j + p.ensembles[1] * (npar - 1)] = rp[s][nc][j]
    totout = sum(len(q.outputs) for q in inp)
    er = np.zeros((totout, max(6, nc1 + 4)))
    em = np.zeros_like(er)
    o = -1
    for s in range(seq):
        p = inp[s]
        for n in p.outputs:
            if p.d_data[n] <= 0:
                continue
            d = np.real(data[s][n]).copy()
            o += 1
            g = list(p.gpoints[n])
            d = freshape(d, g)
            m = min(p.dimensions, len(g) - 2)
            for nd in range(1, m):
                if p.ftransforms[n][nd]:
                    d = np.fft.fftshift(d, axes=nd + 1)
            d, xkn = xcompress(n, d, p, p.xk[n])
            gp = list(d.shape[:-1])
            ddata = int(np.prod(gp))
            d = freshape(d, [ddata, sx])
            mx = np.max(np.abs(d[:, 0])) ** 2                            # :87
            if not (p.relerr and mx > p.tol):
                mx = 1.0
            if ne > 1:
                d[:, sx - 1] = np.abs(np.sqrt((d[:, sx - 1] - d[:, 0] ** 2 + 0j) / n1))  # :95
            else:
                d[:, sx - 1] = 0
            for nc in range(2, p.nchk + p.fbsw + 1):
                d[:, nc - 1] = np.abs(d[:, nc - 1] - d[:, 0])            # :105
                er[o, nc - 1] = np.mean(d[:, nc - 1] ** 2)
                em[o, nc - 1] = math.sqrt(np.max(d[:, nc - 1] ** 2))
            esum = np.sum(d[:, 1:sx] ** 2, axis=1) + 1e-20               # :109
            ept = (esum > p.tol) & (np.abs(d[:, 0]) > p.cutoffs[n])
            if p.compare[n] is not None:                                 # :119
                q = p.copy()
                q.xk = list(p.xk)
                q.xk[n] = xkn
                q = xgrid_out(n, q)
                dif = np.asarray(p.compare[n](q), dtype=float)
                shp = gp
                if dif.ndim < len(shp):
                    dif = dif.reshape(dif.shape + (1,) * (len(shp) - dif.ndim))
                while dif.ndim > len(shp) and dif.shape[-1] == 1:
                    dif = dif[..., 0]
                dif = np.broadcast_to(dif, shp).copy()
                dif = freshape(dif, [ddata, 1])
                d = np.concatenate([d, dif], axis=1)
                ept = ept & (np.abs(d[:, sx]) > p.cutoffs[n])            # :127
                mx = np.max(np.abs(d[:, sx]) ** 2)
                if not (p.relerr and mx > p.tol):
                    mx = 1.0
                dif2 = (d[:, 0] - d[:, sx]) ** 2                         # :136
                em[o, sx] = math.sqrt(np.max(dif2) / mx)
                er[o, sx] = np.mean(dif2) / mx
                if ne > 1:
                    er[o, sx + 1] = np.sum(ept * (dif2 / esum))          # :140
                er[o, sx + 2] = np.sum(ept)
            er[o, 1:p.nchk] = er[o, 1:p.nchk] / mx                       # :144
            er[o, sx - 1] = np.mean(d[:, sx - 1] ** 2) / mx              # :146
            em[o, sx - 1] = math.sqrt(np.max(d[:, sx - 1] ** 2) / mx)
            nz = np.sum(er[o, 1:sx + 1] > 0)
            er[o, 0] = np.sum(er[o, 1:sx + 1]) / (1e-99 + nz)            # :148
            er[o, 0:sx + 1] = np.sqrt(er[o, 0:sx + 1])                   # :149
            data[s][n] = d
    error = np.zeros(max(6, sx + 4))
    for c in range(1, sx + 1):                                           # :181-184
        pts = 1e-99 + np.sum(er[:, c] > p.tol)
        error[c] = math.sqrt(np.sum(er[:, c] ** 2) / pts)
    error[0] = math.sqrt(np.sum(error[1:sx + 1] ** 2) / (1e-99 + np.sum(error[1:sx + 1] > p.tol)))
    error[sx + 1:sx + 3] = np.sum(er[:, sx + 1:sx + 3], axis=0)
    error[sx + 1] = error[sx + 1] / (1e-20 + error[sx + 2])
    error[sx + 2] = time.perf_counter() - t0
    if any(q.rawdata for q in inp):
        return error, data, inp, raw                                     # xsim.m:1 [error,data,input,raw]
    return error, data, inp
