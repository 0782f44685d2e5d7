"""Build xs_problem structs for the C ABI tests."""
import ctypes

from xspde_matlab_b200 import _lib


def make_problem(dimensions=2, fields=1, noises=2, inrandoms=0, points=(51, 64), ranges=(1.0, 10.0), steps=4,
                 checks=1, ensembles=(128, 8, 1), method=0, precision=0, seed=0,
                 deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
                 initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2",
                 observe=("@(a,p) a.*conj(a)", "@(a,p) real(a)"), params=None, boundaries=None):
    p = _lib.XsProblem()
    keep = []
    p.dimensions = dimensions
    p.fields = fields
    p.noises = noises
    p.inrandoms = inrandoms
    points = list(points)[:dimensions]
    ranges = list(ranges)[:dimensions]
    for i in range(dimensions):
        p.points[i] = points[i]
        p.ranges[i] = ranges[i]
        p.origins[i] = 0.0 if i == 0 else -ranges[i] / 2
    p.steps = steps
    p.checks = checks
    for i, e in enumerate(ensembles):
        p.ensembles[i] = e
    p.method = method
    p.iterations = 4
    p.ipsteps = 2 if method in (0, 1) else 1
    p.precision = precision
    p.seed = seed
    p.deriv = deriv.encode()
    p.initial = initial.encode()
    p.linear = linear.encode() if linear else None
    obs = (ctypes.c_char_p * len(observe))(*[o.encode() for o in observe])
    keep.append(obs)
    p.nobserve = len(observe)
    p.observe = obs
    if params:
        names = list(params)
        nm = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
        vals = (ctypes.c_double * len(names))(*[float(params[n]) for n in names])
        keep += [nm, vals]
        p.nparams = len(names)
        p.param_names = nm
        p.param_values = vals
    if boundaries is not None:
        flat = [int(x) for x in boundaries]
        arr = (ctypes.c_int * len(flat))(*flat)
        keep.append(arr)
        p.boundaries = arr
    return p, keep
