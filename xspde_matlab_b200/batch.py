"""Uneven batch: many independent xSPDE inputs integrated by one CUDA-graph launch.

The reference runs one input at a time (Simulator/xsim.m:44-60 loops over
sequences; Simulator/xensemble.m:25-108 over blocks), so a sweep of hundreds
of small problems pays one MATLAB time loop each.  Here every input becomes an
item of an ``xs_batch`` (include/xspde_b200.h): items whose generated kernels
agree share a persistent kernel with a longest-first work queue, items too
large for shared memory run their streaming launches inside the same graph,
and the project's autotuner picks each variant's trajectory tile.

An item is one ensemble block (``ensembles = [ntraj, 1, 1]``); its result is
the block mean of every observable, exactly what ``GpuPath.run_path(0, 1, 1)``
returns for the same input.  With ``checks = 1`` the graph also runs the
coarse pass (``run_path(0, 1, 2)``), and ``results`` returns the fine pass
(Richardson-extrapolated when ``order > 0``) with the step error beside it, as
xsim forms them (Simulator/xensemble.m:41-45, xsim.m:64-98).
"""
import ctypes

import numpy as np

from . import _lib
from .xsim import make_problem, xpreferences

DRIFTS = {
    # cubic NLS with multiplicative (phase) noise: da = i|a|^2 a dt + i g a dW
    "nls": dict(deriv="@(a,w,p) 1i*abs(a).^2.*a + 1i*p.g*a.*w(1,:)",
                linear1="@(p) 0.5i*p.Dx.^2", linear2="@(p) 0.5i*(p.Dx.^2+p.Dy.^2)",
                initial1="@(v,p) exp(-p.x.^2/4) + 0*v(1,:)",
                initial2="@(v,p) exp(-(p.x.^2+p.y.^2)/4) + 0*v(1,:)"),
    # Allen-Cahn with multiplicative noise: da = (a - a^3) dt + g a dW
    "allen_cahn": dict(deriv="@(a,w,p) a - a.^3 + p.g*a.*w(1,:)",
                       linear1="@(p) 0.05*p.Dx.^2", linear2="@(p) 0.05*(p.Dx.^2+p.Dy.^2)",
                       initial1="@(v,p) 0.2*v(1,:)", initial2="@(v,p) 0.2*v(1,:)"),
}


def uneven_instances(n=512, seed=1, output_points=5):
    """The uneven-batch workload: n inputs drawn with a Philox generator of the
    given seed.  Each is 1D (N in {32, ..., 1024}) or 2D (N x N, N in
    {32, 64, 128, 256}) on a periodic box of side 20, with cubic-NLS or
    Allen-Cahn drift, multiplicative noise amplitude g ~ U[0.001, 0.1], total
    steps ~ U{50..2000} (split over output_points - 1 output intervals of
    t in [0, 1]), 64..1024 trajectories (multiples of 64), FP32 fields, MP."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    intervals = output_points - 1
    for i in range(n):
        two_d = bool(rng.integers(0, 2))
        N = int(2 ** rng.integers(5, 9)) if two_d else int(2 ** rng.integers(5, 11))
        drift = "nls" if rng.integers(0, 2) == 0 else "allen_cahn"
        g = float(rng.uniform(0.001, 0.1))
        steps = int(rng.integers(50, 2001))
        ntraj = 64 * int(rng.integers(1, 17))
        d = DRIFTS[drift]
        dim = 2 if two_d else 1
        out.append(dict(
            name="%s_%dd_%d" % (drift, dim, N), drift=drift,
            dimensions=dim + 1, fields=1, noises=1, inrandoms=1,
            points=[output_points] + [N] * dim, ranges=[1.0] + [20.0] * dim,
            steps=max(1, round(steps / intervals)), checks=0, ensembles=[ntraj, 1, 1],
            method="MP", precision="fp32", seed=i + 1, g=g,
            deriv=d["deriv"], linear=d["linear%d" % dim], initial=d["initial%d" % dim],
            observe=["@(a,p) abs(a).^2"]))
    return out


def dpo_instances(blocks=8, ntraj=125000, seed=1, precision="fp64"):
    """Positive-P DPO sweep: `blocks` items of `ntraj` trajectories, each with
    its own pump eps ~ U[0.5, 2] (numpy Philox generator of the given seed) and
    Philox noise seed; 2000 MP steps to t = 10 (problems.DPO_0D)."""
    from .problems import DPO_0D
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for b in range(blocks):
        eps = float(rng.uniform(0.5, 2.0))
        d = dict(DPO_0D, ensembles=[ntraj, 1, 1], seed=b + 1, precision=precision, name="dpo_0d",
                 params=dict(DPO_0D["params"], eps=eps))
        out.append(d)
    return out


def trajectory_steps(inp):
    """Trajectory-steps of one input: ntraj x steps x (points(1) - 1)."""
    return inp["ensembles"][0] * inp["steps"] * max(1, inp["points"][0] - 1)


class Batch:
    """One ``xs_batch`` over xSPDE inputs (dicts as for ``xsim``)."""

    def __init__(self, inputs, skip_unsupported=False):
        L = _lib.lib()
        self.skipped = []
        prefs = []
        for k, inp in enumerate(inputs):
            p = xpreferences(_named_scalars(inp))[0]
            if skip_unsupported and not _supported(p):
                self.skipped.append(k)
                continue
            prefs.append((k, p))
        self.index = [k for k, _ in prefs]
        self.inputs = [p for _, p in prefs]
        if not self.inputs:
            raise ValueError("no supported items in the batch")
        built = [make_problem(p, 0, runtime_params=True) for p in self.inputs]
        self._keep = [kp for _, kp in built]
        arr = (_lib.XsProblem * len(built))(*[pr for pr, _ in built])
        self._arr = arr
        h = ctypes.c_void_p()
        _lib.check(L.xs_batch_create(ctypes.cast(arr, ctypes.c_void_p), len(built), ctypes.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.lib().xs_batch_destroy(h)
            except Exception:
                pass
            self.h = None

    def __len__(self):
        return len(self.inputs)

    def tune(self, mode=1):
        """Pick each variant's tile (mode 1 times the candidates on the GPU)."""
        _lib.check(_lib.lib().xs_batch_tune(self.h, mode))

    def run(self, stream=None):
        """Launch the whole batch (one CUDA graph; captured on the first call)."""
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _lib.check(_lib.lib().xs_batch_run(self.h, st))

    def sync(self):
        _lib.check(_lib.lib().xs_batch_sync(self.h))

    def summary(self):
        """{items, variants, streaming items, kernel launches per run}."""
        info = (ctypes.c_int * 4)()
        _lib.check(_lib.lib().xs_batch_info(self.h, -1, info, 4))
        return dict(items=info[0], variants=info[1], streaming=info[2], launches=info[3])

    def info(self, i):
        """Tile of item i: variant, path (1 resident, 2 streaming), G, threads, CTAs, units."""
        info = (ctypes.c_int * 6)()
        _lib.check(_lib.lib().xs_batch_info(self.h, i, info, 6))
        return dict(variant=info[0], path=info[1], G=info[2], threads=info[3], ctas=info[4], units=info[5])

    def passes(self, i):
        """Block means of item i per check pass: [fine] or, with checks = 1,
        [fine, coarse]; each a list with one complex array per observable,
        shaped [lines, points(1), space...] like GpuPath.run_path's av."""
        L = _lib.lib()
        n = L.xs_batch_av_doubles(self.h, i)
        buf = np.empty(max(n, 1), dtype=np.float64)
        _lib.check(L.xs_batch_results(self.h, i, buf.ctypes.data))
        cbuf = buf[:n].view(np.complex128)
        p = self.inputs[i]
        out, pos = [], 0
        for _ in range(1 + (1 if p.checks[0] else 0)):
            one = []
            for o in range(len(p.observe)):
                shp = _obs_shape(p, o)
                m = int(np.prod(shp))
                one.append(np.reshape(cbuf[pos:pos + m], shp, order="F"))
                pos += m
            out.append(one)
        return out

    def results(self, i, step_error=False):
        """Block means of item i: one complex array per observable, shaped
        [lines, points(1), space...] like GpuPath.run_path's av.  With
        checks = 1 the fine pass, extrapolated as d1 + (d1 - d2)/(2^order - 1)
        when order > 0 (xsim's _ensembles); step_error=True also returns the
        step errors |mean - d2| per observable (None without checks)."""
        ps = self.passes(i)
        p = self.inputs[i]
        if len(ps) == 1:
            return (ps[0], None) if step_error else ps[0]
        fine, coarse = ps
        if p.order > 0:
            mean = [d1 + (d1 - d2) / (2 ** p.order - 1.0) for d1, d2 in zip(fine, coarse)]
            ref = fine
        else:
            mean, ref = fine, coarse
        if not step_error:
            return mean
        return mean, [np.abs(m - r) for m, r in zip(mean, ref)]


def _named_scalars(inp):
    """Move the workload's named scalars (p.g) into the input's params."""
    d = dict(inp)
    params = dict(d.pop("params", {}) or {})
    for k in ("g",):
        if k in d:
            params[k] = d.pop(k)
    d.pop("name", None)
    d.pop("drift", None)
    d["params"] = params
    return d


def _obs_shape(p, o):
    """[lines, points(1), space...] of observable o; site observables keep the space axes."""
    lines, spatial = _obs_info(p, o)
    return (lines, p.points[0]) + (tuple(p.space) if spatial else ())


_OBS_CACHE = {}


def _obs_info(p, o):
    """(lines, spatial) of observable o, from a compile-only handle of the input."""
    key = (p.observe[o], p.dimensions, p.fields)
    if key not in _OBS_CACHE:
        L = _lib.lib()
        pr, keep = make_problem(p, 0, runtime_params=True)
        h = ctypes.c_void_p()
        _lib.check(L.xs_create(ctypes.byref(pr), ctypes.byref(h)))
        try:
            ln, sp = ctypes.c_int(), ctypes.c_int()
            _lib.check(L.xs_observe_info(h, o, ctypes.byref(ln), ctypes.byref(sp)))
            _OBS_CACHE[key] = (ln.value, bool(sp.value))
        finally:
            L.xs_destroy(h)
    return _OBS_CACHE[key]


def _supported(p):
    """True when the library accepts the input as a batch item (host check only)."""
    pr, keep = make_problem(p, 0, runtime_params=True)
    arr = (_lib.XsProblem * 1)(pr)
    h = ctypes.c_void_p()
    code = _lib.lib().xs_batch_create(ctypes.cast(arr, ctypes.c_void_p), 1, ctypes.byref(h))
    if code == _lib.XS_OK:
        _lib.lib().xs_batch_destroy(h)
        return True
    return False
