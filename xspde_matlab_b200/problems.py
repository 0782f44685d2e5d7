"""The benchmark problems as xSPDE input structs.

snls_1d: 1D stochastic NLS, 64 points on [-5,5], da/dt = i d2a/dx2 +
  i|a|^2 a + 0.01 xi, a0 = exp(-x^2), 1024 trajectories in 8 blocks, 200 steps
  to t = 1 (50 steps x 4 substeps between 51 output points).
gpe_2d: 2D stochastic Gross-Pitaevskii / complex Ginzburg-Landau on 256x256
  periodic over [-10,10]^2, da/dt = (i+0.1) lap a + (1-|a|^2) a - 0.5i |a|^2 a
  + 0.05 xi, a0 = 1 + 0.1 complex Gaussian, 4096 trajectories in 16 blocks,
  500 steps to t = 5 (51 output points).
xi is complex white noise (w1 + i w2)/sqrt(2).
"""
import ctypes

from . import _lib
from .xsim import GpuPath, xpreferences

SNLS_1D = dict(
    dimensions=2, points=[51, 64], ranges=[1.0, 10.0], steps=4, ensembles=[128, 8, 1], noises=2, method="RK4",
    checks=0,
    deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
    initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2",
    observe=["@(a,p) a.*conj(a)", "@(a,p) real(a)"])

GPE_2D = dict(
    dimensions=3, points=[51, 256, 256], ranges=[5.0, 20.0, 20.0], steps=10, ensembles=[256, 16, 1], noises=2,
    method="MP", checks=0, precision="fp32",
    deriv="@(a,w,p) (1-abs(a).^2).*a - 0.5i*abs(a).^2.*a + 0.05*(w(1,:)+1i*w(2,:))/sqrt(2)",
    initial="@(v,p) 1 + 0.1*(v(1,:)+1i*v(2,:))/sqrt(2)", linear="@(p) (1i+0.1)*(p.Dx.^2+p.Dy.^2)",
    observe=["@(a,p) abs(a).^2"])

PROBLEMS = {"snls_1d": SNLS_1D, "gpe_2d": GPE_2D}


def compile_check(name, **over):
    """NVRTC-compile the kernels of a named problem for sm_100a (no GPU needed)."""
    p = dict(PROBLEMS[name], **over)
    q = xpreferences([p])[0]
    g = GpuPath.__new__(GpuPath)
    pr, keep = _struct(q)
    log = ctypes.create_string_buffer(1 << 16)
    _lib.check(_lib.lib().xs_compile_check(ctypes.byref(pr), log, len(log)))
    del g, keep
    return log.value.decode(errors="replace")


def _struct(q):
    pr = _lib.XsProblem()
    keep = []
    pr.dimensions, pr.fields, pr.noises, pr.inrandoms = q.dimensions, q.fields, q.noises, q.inrandoms
    for d in range(len(q.points)):
        pr.points[d], pr.ranges[d], pr.origins[d] = q.points[d], q.ranges[d], q.origins[d]
    pr.steps, pr.checks = q.steps[0], q.checks[0]
    for i in range(3):
        pr.ensembles[i] = q.ensembles[i]
    pr.method, pr.iterations, pr.ipsteps = _lib.METHODS[q.method], q.iterations, q.ipsteps
    pr.precision = 1 if q.precision == "fp32" else 0
    pr.seed = q.seed
    pr.deriv, pr.initial = q.deriv.encode(), q.initial.encode()
    pr.linear = (q.get("linear") or "").encode()
    obs = (ctypes.c_char_p * len(q.observe))(*[o.encode() for o in q.observe])
    keep.append(obs)
    pr.nobserve, pr.observe = len(q.observe), obs
    return pr, keep
