"""Host mirror of xSPDE's control layer over the GPU ensemble path.

``xsim(p, ...)`` and ``xspde(p, ...)`` take the reference's input struct (a dict
with the same field names: dimensions, fields, points, ranges, origins, steps,
checks, ensembles, noises, inrandoms, method, iterations, ipsteps, order, seed,
boundaries, linear, deriv, initial, observe, output, compare, axes ...) and
return ``(error, data, input)`` as Simulator/xsim.m:1 does.  Functions that run
on the device -- ``deriv`` (alias ``da``), ``initial``, ``observe``, ``linear``
-- are given as the text of MATLAB anonymous functions; host-side functions
-- ``output``, ``compare`` -- are Python callables, as in the reference where
they run after the ensemble loop (Simulator/xensemble.m:88, xsim.m:121).

The ensemble loop (Simulator/xensemble.m:25-108) calls the GPU's p.path
replacement once per check pass for a group of blocks, then accumulates
block moments and the step-error/sampling-error columns exactly as the
reference does.  There is no CPU fallback: a problem the device path cannot
run raises ``XsError``.
"""
import ctypes
import math
import time

import numpy as np

from . import _lib

__all__ = ["xpreferences", "xsim", "xspde", "GpuPath", "Struct"]


class Struct(dict):
    """Attribute-access dict standing in for a MATLAB struct."""

    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError as exc:
            raise AttributeError(k) from exc

    def __setattr__(self, k, v):
        self[k] = v

    def copy(self):
        return Struct(self)


_METHOD_ALIASES = {"xRK4": "RK4", "xMP": "MP", "xEuler": "Euler", "xRK2": "RK2", "xImplicit": "Implicit"}


def _vec(v, n, fill):
    v = [] if v is None else list(np.atleast_1d(v))
    return v + [fill] * (n - len(v))


def _fsize(a):
    """MATLAB size: trailing singletons dropped (at least two entries)."""
    s = list(np.shape(a))
    while len(s) > 2 and s[-1] == 1:
        s.pop()
    return s + [1] * (2 - len(s))


def xpreferences(inputs):
    """Defaults of Simulator/xpreferences.m:11-414 for the fields this path uses."""
    if isinstance(inputs, dict):
        inputs = [inputs]
    out = []
    origin = 0.0
    for s, pin in enumerate(inputs):
        p = Struct(pin)
        if "da" in p and "deriv" not in p:
            p.deriv = p.da
        if "step" in p and "method" not in p:
            p.method = p.step
        p.ensembles = [int(x) for x in _vec(p.get("ensembles"), 3, 1)]
        p.tol = float(p.get("tol", 1e-20))
        p.dimensions = int(p.get("dimensions", 1))
        nd = max(1, p.dimensions)
        p.fields = int(np.atleast_1d(p.get("fields", 1))[0])
        dflt = [51] + [35] * (nd - 1)
        pts = [int(x) for x in np.atleast_1d(p.get("points", dflt))]
        pts = pts + dflt[len(pts):]
        chk = [int(x) for x in np.atleast_1d(p.get("checks", [1] + [0] * (nd - 1)))]
        p.checks = chk + [0] * (nd - len(chk))
        if s > 0:
            p.checks = out[0].checks
        if any(p.checks[1:]):
            raise _lib.XsError(-9, "space-step checks (checks(2:end)) are not supported")
        p.iterations = int(p.get("iterations", 4))
        p.rawdata = int(p.get("rawdata", 0))  # xpreferences.m:85
        p.auxfields = int(np.atleast_1d(p.get("auxfields", 0))[0])  # xpreferences.m:46, one auxiliary cell
        # noise and random cells (xpreferences.m:65-76): Gaussian x-space, then k-filtered
        nz, kz = p.get("noises", None), p.get("knoises", None)
        p.knoises = int(np.atleast_1d(kz)[0]) if kz is not None else 0
        p.noises = int(np.atleast_1d(nz)[0]) if nz is not None else (0 if kz is not None else p.fields)
        rz, krz = p.get("inrandoms", None), p.get("krandoms", None)
        p.krandoms = int(np.atleast_1d(krz)[0]) if krz is not None else 0
        p.inrandoms = int(np.atleast_1d(rz)[0]) if rz is not None else (0 if krz is not None else p.noises)
        p.ranges = [float(x) for x in _vec(p.get("ranges", [10.0] * nd), nd, 10.0)]
        st = [int(x) for x in np.atleast_1d(p.get("steps", [1]))]
        p.steps = st + [1] * (nd - len(st))
        org = [origin] + [-r / 2 for r in p.ranges[1:]]
        og = [float(x) for x in np.atleast_1d(p.get("origins", org))]
        p.origins = og + org[len(og):]
        for d in range(1, nd):
            pts[d] = 1 + (pts[d] - 1) * p.steps[d]
        p.points = pts
        p.seed = int(p.get("seed", 0))
        m = p.get("method", None)
        if m is None:
            m = "RK4" if int(np.prod(p.ensembles)) == 1 else "MP"
        if callable(m):
            m = m.__name__
        p.method = _METHOD_ALIASES.get(m, m)
        if p.method not in _lib.METHODS:
            raise _lib.XsError(-9, "method %r is not available on the device path" % (m,))
        p.ipsteps = int(p.get("ipsteps", 1 if p.method in ("Euler", "Implicit", "RK2") else 2))
        p.order = int(p.get("order", 0))
        p.relerr = int(p.get("relerr", 1))
        p.precision = str(p.get("precision", "fp64")).lower()
        for key in ("deriv", "initial", "linear"):
            v = p.get(key, None)
            if v is not None and not isinstance(v, str):
                raise _lib.XsError(-2, "p.%s must be the text of a MATLAB anonymous function" % key)
        obs = p.get("observe", None)
        if obs is None:
            obs = ["@(a,p) a"]
        elif isinstance(obs, str):
            obs = [obs]
        for o in obs:
            if not isinstance(o, str):
                raise _lib.XsError(-2, "p.observe entries must be MATLAB anonymous-function text")
        p.observe = list(obs)
        outs = p.get("output", None)
        outs = [outs] if callable(outs) else list(outs or [])
        outs += [None] * (len(p.observe) - len(outs))
        p.output = [o if o is not None else (lambda o, p, n=n: o[n]) for n, o in enumerate(outs)]
        cmp = p.get("compare", None)
        cmp = [cmp] if callable(cmp) else list(cmp or [])
        p.compare = cmp + [None] * (len(p.output) - len(cmp))
        cut = p.get("cutoff", -1e20)
        p.cutoffs = list(p.get("cutoffs", [])) + [cut] * len(p.output)
        ax = list(p.get("axes", None) or [])
        ax += [None] * (len(p.output) - len(ax))
        p.axes = [list(a) + [0] * (nd + 10 - len(a)) if a is not None else [0] * (nd + 10) for a in ax]
        # p.transforms{n}: Fourier-space observables (xpreferences.m, xnft.m)
        tr = p.get("transforms", None)
        if tr is None:
            tr = [[0] * (nd + 1)] * len(p.observe)
        elif not isinstance(tr, (list, tuple)) or not isinstance(tr[0], (list, tuple, np.ndarray)):
            tr = [tr] if not isinstance(tr, (list, tuple)) else list(tr)
        tr = [[int(v) for v in np.atleast_1d(x)] + [0] * (nd + 1) for x in tr]
        tr += [[0] * (nd + 1)] * (len(p.observe) - len(tr))
        p.transforms = [x[: nd + 1] for x in tr]
        ftr = p.get("ftransforms", None)
        p.ftransforms = [list(x) for x in (ftr if ftr is not None else p.transforms)]
        p.ftransforms += [[0] * (nd + 1)] * (len(p.output) - len(p.ftransforms))
        p.params = dict(p.get("params", {}))
        bnd = p.get("boundaries", None)
        if bnd is not None:
            b = []
            for d in range(1, nd):
                bd = bnd[d] if d < len(bnd) and bnd[d] is not None else None
                b.append(np.zeros((p.fields, 2), int) if bd is None else np.atleast_2d(np.asarray(bd, int)))
            p.boundaries = b if any(np.any(x != 0) for x in b) else None
        else:
            p.boundaries = None
        p.dt = p.ranges[0] / max(1, p.points[0] - 1)
        p.nchk = 1 + sum(p.checks)
        p.dx = [p.ranges[d] / max(1, p.points[d] - 1) if p.points[d] > 1 else 1.0 for d in range(nd)]
        p.dk = [2 * math.pi / (p.points[d] * p.dx[d]) for d in range(nd)]
        p.dk[0] /= p.steps[0]
        p.space = p.points[1:]
        p.nspace = int(np.prod(p.space)) if p.space else 1
        p.xc = [p.origins[d] + np.arange(p.points[d]) * p.dx[d] for d in range(nd)]
        p.kc = [(np.arange(p.points[d]) - p.points[d] // 2) * p.dk[d] for d in range(nd)]
        p.kc[0] = (np.arange(p.points[0]) - p.points[0] // 2) * (2 * math.pi / (p.ranges[0] + p.dt))
        # lattice coordinates for host-side functions (transfer): p.r{d}, p.x, p.y, p.z shaped
        # [1, ..., N_d, ..., 1] like a field array (xgrid.m)
        p.r = [None] * max(4, nd)
        for d in range(1, nd):
            sh = [1] * (nd + 1)
            sh[d] = p.points[d]
            p.r[d] = p.xc[d].reshape(sh)
        p.x, p.y, p.z = p.r[1], p.r[2], p.r[3]
        # k grids in propagation (FFT) order, shaped like p.x (xgrid.m), for p.nfilter / p.rfilter
        p.k = [None] * max(4, nd)
        for d in range(1, nd):
            p.k[d] = np.fft.ifftshift(p.kc[d]).reshape(p.r[d].shape)
        p.kx, p.ky, p.kz = p.k[1], p.k[2], p.k[3]
        p.sequence = s
        p.transfer = p.get("transfer", None)
        out.append(p)
        origin = p.origins[0] + p.ranges[0]
    return out


def _filter_table(fn, nc, p):
    """Factors of a k-space filter (p.nfilter / p.rfilter, Simulator/xnoise.m:42,
    xrandom.m:26) on the FFT-ordered k lattice: fn(ones, p) as [nc][space] complex
    FP64 (interleaved re, im; site index column-major).  The device applies
    filters of the form w .* f(p.kx, ...): a random probe checks that fn is one."""
    shape = [nc] + list(p.space) + [1]
    f = np.broadcast_to(np.asarray(fn(np.ones(shape, complex), p), dtype=complex), shape)
    v = np.random.default_rng(7).normal(size=shape).astype(complex)
    if not np.allclose(np.asarray(fn(v, p), dtype=complex), v * f, rtol=1e-12, atol=1e-300):
        raise ValueError("p.nfilter / p.rfilter must multiply each k-space value by a function of k")
    f = np.reshape(f[..., 0], (nc, -1), order="F")
    return np.ascontiguousarray(f).view(np.float64).reshape(-1)


def make_problem(p, path_kind=0, runtime_params=False):
    """The C-ABI problem struct (xs_problem) of one preference-filled input;
    returns it with the ctypes arrays it points into (keep them alive).
    With runtime_params the named scalars p.<name> are read by the kernels
    at run time instead of being compiled in."""
    pr = _lib.XsProblem()
    pr.dimensions = p.dimensions
    pr.fields = p.fields
    pr.noises = p.noises
    pr.inrandoms = p.inrandoms
    pr.knoises = p.knoises
    pr.krandoms = p.krandoms
    for d in range(len(p.points)):
        pr.points[d] = p.points[d]
        pr.ranges[d] = p.ranges[d]
        pr.origins[d] = p.origins[d]
    pr.steps = p.steps[0]
    pr.checks = p.checks[0]
    for i in range(3):
        pr.ensembles[i] = p.ensembles[i]
    pr.method = _lib.METHODS[p.method]
    pr.iterations = p.iterations
    pr.ipsteps = p.ipsteps
    pr.precision = 1 if p.precision in ("fp32", "single", "float32") else 0
    pr.seed = p.seed & 0xFFFFFFFFFFFFFFFF
    keep = []
    if p.boundaries is not None:
        flat = np.concatenate([np.asarray(b, np.int32).reshape(-1) for b in p.boundaries]).astype(np.int32)
        arr = (ctypes.c_int * flat.size)(*flat.tolist())
        keep.append(arr)
        pr.boundaries = arr
    pr.deriv = (p.get("deriv") or "@(a,w,p) 0*a").encode()
    pr.initial = (p.get("initial") or "@(v,p) 0").encode()
    pr.linear = (p.get("linear") or "").encode()
    pr.auxfields = p.auxfields
    if p.auxfields:
        pr.define = (p.get("define") or "").encode()
    obs = (ctypes.c_char_p * len(p.observe))(*[o.encode() for o in p.observe])
    keep.append(obs)
    pr.nobserve = len(p.observe)
    pr.observe = obs
    names = list(p.params.keys())
    if names:
        nm = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
        vals = (ctypes.c_double * len(names))(*[float(p.params[n]) for n in names])
        keep += [nm, vals]
        pr.nparams = len(names)
        pr.param_names = nm
        pr.param_values = vals
    pr.path_kind = path_kind
    pr.runtime_params = 1 if runtime_params else 0
    pr.sequence = int(p.get("sequence", 0) or 0)
    pr.boundary_values = 1 if callable(p.get("boundfun", None)) else 0
    for nc, key in ((p.knoises, "nfilter"), (p.krandoms, "rfilter")):
        fn = p.get(key, None)
        if nc > 0 and fn is not None:
            tab = _filter_table(fn, nc, p)
            arr = (ctypes.c_double * tab.size)(*tab.tolist())
            keep.append(arr)
            setattr(pr, key, arr)
    if any(any(t[1:]) or t[0] for t in p.transforms):
        flags = []
        for t in p.transforms:
            flags += [int(t[j]) if j < len(t) else 0 for j in range(4)]
        arr = (ctypes.c_int * len(flags))(*flags)
        keep.append(arr)
        pr.transforms = arr
    return pr, keep


class GpuPath:
    """One compiled device problem: the p.path/p.method replacements of one input."""

    def __init__(self, p, path_kind=0, runtime_params=False):
        L = _lib.lib()
        pr, keep = make_problem(p, path_kind, runtime_params)
        h = ctypes.c_void_p()
        _lib.check(L.xs_create(ctypes.byref(pr), ctypes.byref(h)))
        self._keep = keep
        self.h = h
        self.p = p
        self.obs = []
        for o in range(len(p.observe)):
            ln, sp = ctypes.c_int(), ctypes.c_int()
            _lib.check(L.xs_observe_info(h, o, ctypes.byref(ln), ctypes.byref(sp)))
            dims = (ctypes.c_int * 3)()
            _lib.check(L.xs_observe_shape(h, o, dims))
            shape = tuple(dims[d] for d in range(len(p.space)))  # 1 where a partial Int/Ave reduces
            self.obs.append((ln.value, bool(sp.value), shape))
        self.per_block = L.xs_av_doubles_per_block(h)
        # 1 resident, 2 streaming 2D, 3 streaming 3D (xs_path_kind)
        self.kind = L.xs_path_kind(h)

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.lib().xs_destroy(h)
            except Exception:
                pass
            self.h = None

    def av_shapes(self):
        P = self.p
        return [(ln, P.points[0]) + (shape if sp else ()) for ln, sp, shape in self.obs]

    def _boundary_values(self, nc):
        """p.boundfun(a, c, d, p) tabulated at every half step t0 + k dtr/2 of check
        pass nc (the times xprop/xsetbound query in MP, Applications/SDE/MP.m:11-26),
        as complex [times][space dims][fields][2]; handed to the device once per pass."""
        cache = self.__dict__.setdefault("_bv_done", set())
        if nc in cache:
            return
        P = self.p
        fine = P.checks[0] and nc != 2
        dtr = P.dt / (2 * P.steps[0]) if fine else P.dt / P.steps[0]
        nsteps = (P.points[0] * P.steps[0] - 1) * (2 if fine else 1)
        ntimes = 2 * nsteps + 3
        nd = P.dimensions - 1
        tab = np.zeros((ntimes, nd, P.fields, 2), dtype=np.complex128)
        q = P.copy()
        for k in range(ntimes):
            q.t = P.origins[0] + k * dtr / 2
            for d in range(nd):
                if P.boundaries is not None and np.any(np.asarray(P.boundaries[d]) != 0):
                    b = np.asarray(P.boundfun(None, 0, d + 1, q), dtype=np.complex128)
                    tab[k, d] = np.broadcast_to(b.reshape(-1, 2) if b.size >= 2 else b, (P.fields, 2))
        tab = np.ascontiguousarray(tab)
        _lib.check(_lib.lib().xs_set_boundary_values(self.h, nc, ntimes, tab.ctypes.data))
        cache.add(nc)

    def run_path(self, first_block, nblocks, nc, a_in=None, a_out=False, raw=False):
        """p.path for blocks [first_block, first_block+nblocks): returns
        (av, a) with av[b][o] complex arrays of shape av_shapes()[o]; with
        raw=True (p.rawdata, Simulator/xpath.m:73-78) also the field at every
        output time, [fields, points(1), space..., ens1*nblocks]: (av, a, raw)."""
        P = self.p
        if callable(P.get("boundfun", None)):
            self._boundary_values(nc)
        buf = np.empty(nblocks * self.per_block, dtype=np.float64)
        ain = None
        if a_in is not None:
            ain = np.asfortranarray(np.asarray(a_in, dtype=np.complex128))
        aout = None
        if a_out:
            aout = np.empty([P.fields] + list(P.space) + [P.ensembles[0] * nblocks], dtype=np.complex128, order="F")
        rout = None
        if raw:
            rout = np.empty([P.fields, P.points[0]] + list(P.space) + [P.ensembles[0] * nblocks],
                            dtype=np.complex128, order="F")
        _lib.check(_lib.lib().xs_run_path_raw(self.h, first_block, nblocks, nc,
                                              ain.ctypes.data if ain is not None else None,
                                              buf.ctypes.data, aout.ctypes.data if aout is not None else None,
                                              rout.ctypes.data if rout is not None else None))
        cbuf = buf.view(np.complex128)
        av, pos = [], 0
        for b in range(nblocks):
            row = []
            for shp in self.av_shapes():
                n = int(np.prod(shp))
                row.append(np.reshape(cbuf[pos:pos + n], shp, order="F"))
                pos += n
            av.append(row)
        if raw:
            return av, aout, rout
        return av, aout


def _hook_methods():
    """p.noisegen / p.randomgen / p.method replacements on a GpuPath."""

    def noise(self, block, draw, scale):
        """One p.noisegen draw (Simulator/xnoise.m:29-32) before any coarse
        averaging: [noises, space..., ens1] real."""
        P = self.p
        out = np.empty([P.noises] + list(P.space) + [P.ensembles[0]], dtype=np.float64, order="F")
        _lib.check(_lib.lib().xs_noise(self.h, block, draw, float(scale), out.ctypes.data))
        return out

    def random(self, block):
        """p.randomgen (Simulator/xrandom.m:20-23): [inrandoms, space..., ens1] real."""
        P = self.p
        out = np.empty([P.inrandoms] + list(P.space) + [P.ensembles[0]], dtype=np.float64, order="F")
        _lib.check(_lib.lib().xs_random(self.h, block, out.ctypes.data))
        return out

    def step(self, a, w, t, dtr):
        """p.method(a, w, p) for one block of trajectories: returns the new field."""
        a = np.array(a, dtype=np.complex128, order="F", copy=True)
        wp = None
        if w is not None:
            wp = np.asfortranarray(np.asarray(w, dtype=np.float64))
        _lib.check(_lib.lib().xs_step(self.h, a.ctypes.data, wp.ctypes.data if wp is not None else None,
                                      float(t), float(dtr)))
        return a

    GpuPath.noise = noise
    GpuPath.random = random
    GpuPath.step = step


_hook_methods()


def _xcompress(n, data, p, xk):
    """Axis reduction of an output array (Applications/SPDE/xcompress.m:18-70)."""
    axes = list(p.axes[n])
    x = list(xk)
    d = len(p.gpoints[n]) - 2
    rank = data.ndim
    shp = list(data.shape) + [1] * d
    mid = [1 + v // 2 for v in shp]
    for ax in range(d):
        ind = axes[ax]
        if np.size(x[ax]) > 1:
            if ax + 1 <= p.dimensions and ax < len(p.ftransforms[n]) and p.ftransforms[n][ax]:
                x[ax] = p.kc[ax]  # k axis (xcompress.m:40-42)
            if np.size(ind) == 1:
                ind = int(np.atleast_1d(ind)[0])
                ind = (list(range(1, shp[ax + 1] + 1)) if ind == 0 else [mid[ax + 1]] if ind == -1
                       else [shp[ax + 1]] if ind == -2 else [ind])
            ind = [int(i) for i in np.atleast_1d(ind)]
            if shp[ax + 1] > len(ind):
                data = np.reshape(data, [int(np.prod(shp[:ax + 1])), shp[ax + 1], -1], order="F")[:, [i - 1 for i in ind], :]
                shp[ax + 1] = len(ind)
            else:
                ind = ind[:shp[ax + 1]]
            x[ax] = np.asarray(x[ax])[[i - 1 for i in ind]]
    return np.reshape(data, shp[:rank], order="F"), x


def _grid(xk):
    """Output-grid broadcast coordinates for compare functions (Applications/SPDE/xgrid.m:49-56)."""
    q = Struct()
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


def _kadd(s, c, x):
    """Neumaier's compensated summation (ZAMM 54 (1974) 39-51), elementwise and in
    place: the running sums s and corrections c together hold each total to about
    one rounding of the exact sum; the result is s + c."""
    t = s + x
    c += np.where(np.abs(s) >= np.abs(x), (s - t) + x, (x - t) + s)
    s[...] = t


class _Checkpoint:
    """Block-granular checkpoint of the moment sums (p.checkpoint, a file name; no counterpart
    in the reference, whose xsim.m:207-210 saves only at the end).  Blocks are independent and
    their noise is keyed by the global block index, so the state after a group of blocks is the
    index of the next block with the compensated sums and their compensation terms; a run
    restarted with the same inputs continues from there and returns bit-identical moments.
    Under several ranks each rank keeps its own file (name.rank<r>.npz) for its own blocks."""

    def __init__(self, inp, rank, size, lo, hi, raw):
        name = inp[0].get("checkpoint", None)
        self.path = None
        self.lo = lo
        if not name or not str(name).strip():
            return
        if raw:
            raise ValueError("p.checkpoint cannot be combined with p.rawdata")
        base = str(name)
        if base.endswith(".npz"):
            base = base[:-4]
        self.path = base + (".rank%d" % rank if size > 1 else "") + ".npz"
        # what must match for a saved state to be continued: the text, numeric and list fields of
        # every input (function handles by their text), the block range and the number of ranks
        def plain(v):
            if isinstance(v, (str, int, float, bool)) or v is None:
                return v
            if isinstance(v, (list, tuple)):
                return [plain(x) for x in v]
            if isinstance(v, dict):
                return {k: plain(x) for k, x in sorted(v.items())}
            if isinstance(v, np.ndarray):  # lattices and tables: shape and a digest of the values
                import hashlib
                return ("ndarray", v.shape, hashlib.sha1(np.ascontiguousarray(v).tobytes()).hexdigest()[:16])
            return type(v).__name__
        keys = [sorted((k, plain(v)) for k, v in dict(q).items() if k not in ("checkpoint", "checkpoint_blocks"))
                for q in inp]
        self.sig = repr((keys, lo, hi, size))

    def resume(self, data, comp):
        """The first block to integrate: lo, or the saved next block (restoring the sums)."""
        import os
        if not self.path or not os.path.exists(self.path):
            return self.lo
        with np.load(self.path, allow_pickle=False) as z:
            if str(z["sig"]) != self.sig:
                raise ValueError("p.checkpoint %s was written by a different run" % self.path)
            for key in z.files:
                if key.startswith("data_"):
                    s, o = (int(x) for x in key[5:].split("_"))
                    data[s][o] = z[key].copy()
                    comp[(s, o)] = z["comp_%d_%d" % (s, o)].copy()
            return int(z["next"])

    def save(self, nxt, data, comp):
        import os
        if not self.path:
            return
        arrs = {"sig": np.array(self.sig), "next": np.array(nxt)}
        for s, row in enumerate(data):
            for o, d in enumerate(row):
                if d is not None:
                    arrs["data_%d_%d" % (s, o)] = d
                    arrs["comp_%d_%d" % (s, o)] = comp[(s, o)]
        tmp = self.path[:-4] + ".tmp.npz"
        np.savez(tmp, **arrs)
        os.replace(tmp, self.path)


def _ensembles(inp, paths, rank=0, size=1, reduce=None, raw=None):
    """Block loop, check passes and moments (Simulator/xensemble.m:12-108) with
    all blocks of a pass integrated by one device call.  With size > 1 this
    rank integrates its own contiguous share of the blocks and `reduce` sums
    the moment accumulators over the ranks (Simulator/xsim.m:50-57).  With
    `raw` (nested lists [s][nc-1][k]) the blocks' raw trajectories of inputs
    with p.rawdata are stored at k = j + ens(2) (npar-1) for global block
    (npar-1) + j ens(3) (xensemble.m:26,79; xsim.m:42-57)."""
    from .dist import shard
    p1 = inp[0]
    nb = p1.ensembles[1] * p1.ensembles[2]
    m = p1.nchk
    m1 = max(3, m + 1)
    inv = 1.0 / nb
    data = []
    for s, p in enumerate(inp):
        data.append([None] * len(p.output))
    D = {}
    comp = {}  # compensation terms of the moment sums (_kadd)
    lo, hi = shard(nb, rank, size)
    chunk = max(1, min(nb, int(2 ** 27 // max(1, paths[0].per_block * 8))))
    ckpt = _Checkpoint(inp, rank, size, lo, hi, raw is not None)
    if ckpt.path:
        chunk = max(1, min(chunk, int(p1.get("checkpoint_blocks", chunk))))
    start = ckpt.resume(data, comp)
    failure = None
    try:
        for b0 in range(start, hi, chunk):
            nbk = min(chunk, hi - b0)
            prev = None
            for nc in range(1, p1.nchk + 1):
                prev = None
                for s, p in enumerate(inp):
                    a_in = prev if s > 0 else None
                    if s > 0 and p.transfer is not None:
                        # p.transfer(b, v, p) on the host between the two device paths (xensemble.m:62)
                        if p.inrandoms > 0:
                            v = np.concatenate([paths[s].random(b0 + b) for b in range(nbk)], axis=-1)
                        else:
                            v = np.zeros([0] + list(p.space) + [p.ensembles[0] * nbk])
                        shape = [p.fields] + list(p.space) + [p.ensembles[0] * nbk]
                        r = np.asarray(p.transfer(prev, v, p), dtype=complex)
                        r = r.reshape(r.shape + (1,) * (len(shape) - r.ndim))
                        a_in = np.asfortranarray(np.broadcast_to(r, shape))
                    if raw is not None and p.rawdata:
                        av, prev, r = paths[s].run_path(b0, nbk, nc, a_in=a_in, a_out=(s + 1 < len(inp)), raw=True)
                        e1 = p.ensembles[0]
                        for b in range(nbk):
                            g = b0 + b
                            k = g // p.ensembles[2] + p.ensembles[1] * (g % p.ensembles[2])
                            raw[s][nc - 1][k] = r[..., b * e1:(b + 1) * e1]
                    else:
                        av, prev = paths[s].run_path(b0, nbk, nc, a_in=a_in, a_out=(s + 1 < len(inp)))
                    for b in range(nbk):
                        for o in range(len(p.output)):
                            Dv = np.real(np.asarray(p.output[o](av[b], p)))
                            D[(s, b, nc, o)] = np.reshape(Dv, -1, order="F")
            for s, p in enumerate(inp):
                for b in range(nbk):
                    for o in range(len(p.output)):
                        if p1.checks[0] and p.order > 0:
                            d1, d2 = D[(s, b, 1, o)], D[(s, b, 2, o)]
                            D[(s, b, 2, o)] = d1
                            D[(s, b, 1, o)] = d1 + (d1 - d2) / (2 ** p.order - 1.0)
                        if data[s][o] is None:
                            data[s][o] = np.zeros((D[(s, b, 1, o)].size, m1))
                            comp[(s, o)] = np.zeros_like(data[s][o])
                        ds, dc = data[s][o], comp[(s, o)]
                        for n1 in range(1, m + 1):
                            _kadd(ds[:, n1 - 1], dc[:, n1 - 1], D[(s, b, n1, o)] * inv)
                        _kadd(ds[:, m1 - 1], dc[:, m1 - 1], D[(s, b, 1, o)] ** 2 * inv)
            D.clear()
            ckpt.save(b0 + nbk, data, comp)
    except Exception as ex:
        # a rank that fails still takes part in the reduction below, with a failure
        # count, so that its peers raise at once instead of waiting in the all-reduce
        if size == 1:
            raise
        failure = ex
    for (s, o), c in comp.items():
        data[s][o] = data[s][o] + c
    if size > 1:
        for s, p in enumerate(inp):
            for o in range(len(p.output)):
                if data[s][o] is None:  # a rank without blocks: sizes from the output shapes
                    data[s][o] = np.zeros((int(np.prod(p.gpoints[o][:-1])), m1))
        flat = [x for row in data for x in row] + [np.array([0.0 if failure is None else 1.0])]
        flat = reduce(flat)
        nfail = int(round(float(flat[-1][0])))
        if failure is not None:
            raise failure
        if nfail:
            raise RuntimeError("xsim: %d of %d ranks failed while integrating their ensemble blocks"
                               % (nfail, size))
        pos = 0
        for s in range(len(data)):
            for o in range(len(data[s])):
                data[s][o] = flat[pos]
                pos += 1
    return data


def xsim(*inputs, path_kind=0):
    """Simulate and return (error, data, input) (Simulator/xsim.m:28-214), and
    raw as a fourth value when an input sets p.rawdata: raw[s][nc][k] is the
    [fields, points(1), space..., ens(1)] field array of sequence s, check pass nc
    and ensemble k (xsim.m:42-57; under several ranks each rank holds its own blocks).

    error: [total RMS, step errors..., sampling, difference, chi^2/k, time]
    data[s][o]: columns mean, step error, sampling error, comparison."""
    t0 = time.perf_counter()
    if len(inputs) == 1 and isinstance(inputs[0], (list, tuple)):
        inputs = inputs[0]
    inp = xpreferences(list(inputs))
    paths = [GpuPath(p, path_kind) for p in inp]
    for s, p in enumerate(inp):
        shapes = paths[s].av_shapes()
        O = [np.zeros(x) for x in shapes]
        p.gpoints = []
        for o in range(len(p.output)):
            g = _fsize(p.output[o](O, p))
            p.gpoints.append(g + [max(3, 1 + p.nchk)])
        p.xk = [[p.xc[0]] + [p.xc[d] for d in range(1, len(p.points))] for _ in p.output]
    from .dist import allreduce_sum, world
    rank, size, group = world()
    dev = None
    if size > 1:
        import torch.distributed as tdist
        if tdist.get_backend(group) == "nccl":
            import torch
            dev = torch.device("cuda", torch.cuda.current_device())
    want_raw = any(q.rawdata for q in inp)
    nb = inp[0].ensembles[1] * inp[0].ensembles[2]
    raw = [[[None] * nb for _ in range(inp[0].nchk)] for _ in inp] if want_raw else None
    data = _ensembles(inp, paths, rank, size, reduce=lambda arrs: allreduce_sum(arrs, group, dev), raw=raw)
    p = inp[0]
    ne = p.ensembles[1] * p.ensembles[2]
    sx = max(3, 1 + p.nchk)
    rows = []
    for s, p in enumerate(inp):
        for n in range(len(p.output)):
            d = np.reshape(np.real(data[s][n]), p.gpoints[n], order="F")
            for ax in range(1, min(p.dimensions, len(p.gpoints[n]) - 2)):
                if p.ftransforms[n][ax]:  # k-space axes in centred order (xsim.m:77-81)
                    d = np.fft.fftshift(d, axes=ax + 1)
            d, xkn = _xcompress(n, d, p, p.xk[n])
            gp = list(d.shape[:-1])
            nd_ = int(np.prod(gp))
            d = np.reshape(d, [nd_, sx], order="F")
            er = np.zeros(max(6, p.nchk + 4))
            mx = np.max(np.abs(d[:, 0])) ** 2
            if not (p.relerr and mx > p.tol):
                mx = 1.0
            d[:, sx - 1] = np.abs(np.sqrt((d[:, sx - 1] - d[:, 0] ** 2 + 0j) / (ne - 1))) if ne > 1 else 0.0
            for nc in range(2, p.nchk + 1):
                d[:, nc - 1] = np.abs(d[:, nc - 1] - d[:, 0])
                er[nc - 1] = np.mean(d[:, nc - 1] ** 2)
            esum = np.sum(d[:, 1:sx] ** 2, axis=1) + 1e-20
            ept = (esum > p.tol) & (np.abs(d[:, 0]) > p.cutoffs[n])
            if p.compare[n] is not None:
                dif = np.asarray(p.compare[n](_grid(xkn)), dtype=float)
                if dif.ndim < len(gp):
                    dif = dif.reshape(dif.shape + (1,) * (len(gp) - dif.ndim))
                while dif.ndim > len(gp) and dif.shape[-1] == 1:
                    dif = dif[..., 0]
                dif = np.reshape(np.broadcast_to(dif, gp), [nd_, 1], order="F")
                d = np.concatenate([d, dif], axis=1)
                ept = ept & (np.abs(d[:, sx]) > p.cutoffs[n])
                mx = np.max(np.abs(d[:, sx]) ** 2)
                if not (p.relerr and mx > p.tol):
                    mx = 1.0
                dif2 = (d[:, 0] - d[:, sx]) ** 2
                er[sx] = np.mean(dif2) / mx
                if ne > 1:
                    er[sx + 1] = np.sum(ept * (dif2 / esum))
                er[sx + 2] = np.sum(ept)
            er[1:p.nchk] /= mx
            er[sx - 1] = np.mean(d[:, sx - 1] ** 2) / mx
            er[0] = np.sum(er[1:sx + 1]) / (1e-99 + np.sum(er[1:sx + 1] > 0))
            er[0:sx + 1] = np.sqrt(er[0:sx + 1])
            data[s][n] = d
            rows.append(er)
    er = np.array(rows)
    error = np.zeros(max(6, sx + 4))
    for c in range(1, sx + 1):
        error[c] = math.sqrt(np.sum(er[:, c] ** 2) / (1e-99 + np.sum(er[:, c] > p.tol)))
    error[0] = math.sqrt(np.sum(error[1:sx + 1] ** 2) / (1e-99 + np.sum(error[1:sx + 1] > p.tol)))
    error[sx + 1:sx + 3] = np.sum(er[:, sx + 1:sx + 3], axis=0)
    error[sx + 1] /= 1e-20 + error[sx + 2]
    error[sx + 2] = time.perf_counter() - t0
    fname = inp[0].get("file", None)
    if fname and str(fname).strip():
        save_mat(str(fname), error, data, inp, raw)
    if want_raw:
        return error, data, inp, raw
    return error, data, inp


def _cell(items):
    """A 1 x n MATLAB cell array (object array) of the given values."""
    c = np.empty((1, len(items)), dtype=object)
    for i, v in enumerate(items):
        c[0, i] = v
    return c


# numeric and text input fields kept in the saved input structs (function handles are not)
_SAVED_FIELDS = ("name", "dimensions", "fields", "noises", "knoises", "inrandoms", "krandoms", "auxfields",
                 "points", "ranges", "origins", "steps", "checks", "ensembles", "order", "seed", "method",
                 "iterations", "dt", "dx", "dk", "transforms")


def save_mat(fname, error, data, inp, raw=None):
    """xsim's MATLAB file (Simulator/xsim.m:207-210: save(file, 'error', 'data',
    'input', 'raw')): error as a row vector, data{s}{n} as nested cells, input{s}
    as structs of the numeric and text inputs, raw{s, nc, k} when recorded."""
    import scipy.io
    structs = []
    for p in inp:
        d = {}
        for k in _SAVED_FIELDS:
            v = p.get(k, None)
            if v is None or callable(v):
                continue
            if k == "transforms":
                v = _cell([np.asarray(t, dtype=float) for t in v])
            elif not isinstance(v, str):
                v = np.asarray(v, dtype=float)
            d[k] = v
        structs.append(d)
    out = {"error": np.asarray(error, dtype=float)[None, :],
           "data": _cell([_cell([np.asarray(x) for x in row]) for row in data]),
           "input": _cell(structs)}
    if raw is not None:
        cells = np.empty((len(raw), len(raw[0]), len(raw[0][0])), dtype=object)
        for s, per_s in enumerate(raw):
            for nc, per_nc in enumerate(per_s):
                for k, r in enumerate(per_nc):
                    cells[s, nc, k] = np.zeros(0) if r is None else np.asarray(r)
        out["raw"] = cells
    scipy.io.savemat(fname, out, do_compression=False)


def xspde(*inputs, **kw):
    """xSPDE control function without graphics (Simulator/xspde.m:8)."""
    return xsim(*inputs, **kw)
