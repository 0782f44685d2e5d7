"""The benchmark problems as xSPDE input structs.

snls_1d: 1D stochastic NLS, 64 points on [-5,5], da/dt = i d2a/dx2 +
  i|a|^2 a + 0.01 xi, a0 = exp(-x^2), 1024 trajectories in 8 blocks, 200 steps
  to t = 1 (50 steps x 4 substeps between 51 output points).
gpe_2d: 2D stochastic Gross-Pitaevskii / complex Ginzburg-Landau on 256x256
  periodic over [-10,10]^2, da/dt = (i+0.1) lap a + (1-|a|^2) a - 0.5i |a|^2 a
  + 0.05 xi, a0 = 1 + 0.1 complex Gaussian, 4096 trajectories in 16 blocks,
  500 steps to t = 5 (51 output points).
dpo_0d: positive-P degenerate parametric oscillator, two complex fields
  (alpha, beta), d alpha = (-gam alpha + eps beta - chi alpha^2 beta) dt +
  sqrt(-chi alpha^2) dW1 and the partner equation, gam = 1, chi = 1e-3, eps a
  runtime scalar; MP integrates in the Stratonovich sense, so the drift carries
  the correction -1/2 B dB/dalpha = +chi alpha / 2 (the Ito form is the one
  Euler takes).  alpha = beta = 1 at t = 0; 2000 steps to t = 10.
ac_3d: 3D stochastic Allen-Cahn on 64^3 over [-10,10]^3, da/dt = 0.05 lap a +
  a - a^3 + 0.1 w, Neumann (DCT-I) boundaries in x, Dirichlet (DST-I) in y,
  Neumann at z_min / Dirichlet at z_max (DCT-III/II) in z (xSPDE's flags: 1
  Dirichlet, -1 Neumann), a0 = 0.1 v, FP32 fields, 256
  trajectories in 8 blocks, 100 MP steps to t = 1 (6 output points).
xi is complex white noise (w1 + i w2)/sqrt(2).
"""
import ctypes

from . import _lib
from .xsim import make_problem, xpreferences

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

DPO_0D = dict(
    dimensions=1, fields=2, noises=2, inrandoms=0, points=[11], ranges=[10.0], steps=200, ensembles=[125000, 8, 1],
    method="MP", checks=0, params={"gam": 1.0, "eps": 1.5, "chi": 1e-3},
    deriv="@(a,w,p) [-p.gam*a(1,:)+p.eps*a(2,:)-p.chi*a(1,:).^2.*a(2,:)+0.5*p.chi*a(1,:)"
          "+sqrt(-p.chi*a(1,:).^2).*w(1,:); -p.gam*a(2,:)+p.eps*a(1,:)-p.chi*a(2,:).^2.*a(1,:)"
          "+0.5*p.chi*a(2,:)+sqrt(-p.chi*a(2,:).^2).*w(2,:)]",
    initial="@(v,p) [1; 1]",
    observe=["@(a,p) real(a(1,:).*a(2,:))", "@(a,p) real(a(1,:))"])

AC_3D = dict(
    dimensions=4, points=[6, 64, 64, 64], ranges=[1.0, 20.0, 20.0, 20.0], steps=20, ensembles=[32, 8, 1],
    noises=1, inrandoms=1, method="MP", checks=0, precision="fp32",
    boundaries=[None, [[-1, -1]], [[1, 1]], [[-1, 1]]],
    deriv="@(a,w,p) a - a.^3 + 0.1*w(1,:)", initial="@(v,p) 0.1*v(1,:)",
    linear="@(p) 0.05*(p.Dx.^2+p.Dy.^2+p.Dz.^2)",
    observe=["@(a,p) abs(a).^2", "@(a,p) Int(real(a).^2, p)"])

PROBLEMS = {"snls_1d": SNLS_1D, "gpe_2d": GPE_2D, "dpo_0d": DPO_0D, "ac_3d": AC_3D}


def compile_check(name, **over):
    """NVRTC-compile the kernels of a named problem for sm_100a (no GPU needed)."""
    p = dict(PROBLEMS[name], **over)
    q = xpreferences([p])[0]
    pr, keep = make_problem(q)
    log = ctypes.create_string_buffer(1 << 16)
    _lib.check(_lib.lib().xs_compile_check(ctypes.byref(pr), log, len(log)))
    del keep
    return log.value.decode(errors="replace")
