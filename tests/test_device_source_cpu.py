"""Device code compiled on the host, without a GPU: the functions the expression compiler
generates for a drift and the kernels' Philox/Box-Muller noise, built with g++ from the
kernels' own sources (the device prelude, the noise header and the NVRTC source the library
generates for a problem) with host stand-ins for the few CUDA intrinsics they use.

The generated drift is checked against NumPy evaluating the same MATLAB expressions with
MATLAB's rules: sqrt, log and fractional powers of negative reals return complex values,
round takes halves away from zero, mod takes the sign of the divisor and rem that of the
dividend, sign(z) = z/|z|, comparisons and logical operators give 0 or 1.  The noise is checked
against the oracle's Philox stream (oracle/philox.py) for every counter layout the kernels use:
plain sites, paired sites (x, x + N1/2) and the k-space stream.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest
from scipy.special import erf

from oracle import philox

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KERNELS = os.path.join(ROOT, "xspde_matlab_b200", "csrc", "kernels")

SHIM = r"""
#include <cmath>
#include <cstring>
#define __device__
#define __forceinline__ inline
#define __restrict__
#define __align__(n) alignas(n)
struct uint4 { unsigned x, y, z, w; };
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { uint4 r = {x, y, z, w}; return r; }
inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __logf(float x) { return std::log(x); }
inline void __sincosf(float x, float* s, float* c) { *s = std::sin(x); *c = std::cos(x); }
inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
inline void sincospi(double x, double* s, double* c) { *s = std::sin(M_PI * x); *c = std::cos(M_PI * x); }
inline void sincos(float x, float* s, float* c) { *s = std::sin(x); *c = std::cos(x); }
inline double __shfl_xor_sync(unsigned, double v, int) { return v; }
using namespace std;
"""

# (MATLAB expression in a(k,:) and w, NumPy evaluation of it on z = a(k,:), w1, w2)


def _mround(x):
    return np.where(x >= 0, np.floor(x + 0.5), -np.floor(-x + 0.5))


def _mmod(x, y):
    """MATLAB's mod(x, y) = x - floor(x./y).*y (with the rounded quotient, so an exact
    multiple such as mod(-3.5, 0.7) gives 0 where a remainder without rounding, like
    NumPy's, gives 0.7)."""
    return x - np.floor(x / y) * y


def _mrem(x, y):
    """MATLAB's rem(x, y) = x - fix(x./y).*y."""
    return x - np.trunc(x / y) * y


CASES = [
    ("sqrt(-abs(a(K,:)).^2)", lambda z, w1, w2: np.sqrt(-abs(z) ** 2 + 0j)),
    ("log(real(a(K,:)))", lambda z, w1, w2: np.log(z.real + 0j)),
    ("real(a(K,:)).^0.5", lambda z, w1, w2: (z.real + 0j) ** 0.5),
    ("mod(real(a(K,:)), 0.7) + 1i*rem(imag(a(K,:)), 0.7)",
     lambda z, w1, w2: _mmod(z.real, 0.7) + 1j * _mrem(z.imag, 0.7)),
    ("sign(a(K,:)) + sign(real(a(K,:)))", lambda z, w1, w2: z / abs(z) + np.sign(z.real)),
    ("round(real(a(K,:))) + 1i*fix(3*imag(a(K,:)))", lambda z, w1, w2: _mround(z.real) + 1j * np.trunc(3 * z.imag)),
    ("atan2(imag(a(K,:)), real(a(K,:))) + angle(a(K,:)).^2 + angle(real(a(K,:)))",
     lambda z, w1, w2: np.arctan2(z.imag, z.real) + np.angle(z) ** 2 + np.angle(z.real)),
    ("sech(a(K,:)) + tanh(a(K,:)) + coth(real(a(K,:)))",
     lambda z, w1, w2: 1 / np.cosh(z) + np.tanh(z) + 1 / np.tanh(z.real)),
    ("(real(a(K,:)) > 0).*a(K,:) + (abs(a(K,:)) <= 1).*conj(a(K,:))",
     lambda z, w1, w2: (z.real > 0) * z + (abs(z) <= 1) * np.conj(z)),
    ("a(K,:).^3 - a(K,:).^-2 + 2.^a(K,:)", lambda z, w1, w2: z ** 3 - z ** -2.0 + 2.0 ** z),
    ("exp(1i*a(K,:))./(1 + a(K,:).*conj(a(K,:)))", lambda z, w1, w2: np.exp(1j * z) / (1 + abs(z) ** 2)),
    ("asin(a(K,:)) + acos(a(K,:))/2 + atan(a(K,:))/3",
     lambda z, w1, w2: np.arcsin(z) + np.arccos(z) / 2 + np.arctan(z) / 3),
    ("min(real(a(K,:)), imag(a(K,:))) + max(real(a(K,:)), 0.1)",
     lambda z, w1, w2: np.minimum(z.real, z.imag) + np.maximum(z.real, 0.1)),
    ("erf(real(a(K,:))) + floor(2*imag(a(K,:))) - ceil(real(a(K,:)))",
     lambda z, w1, w2: erf(z.real) + np.floor(2 * z.imag) - np.ceil(z.real)),
    ("sqrt(-0.5*a(K,:).^2).*w(1,:) + cosh(a(K,:)).*w(2,:)",
     lambda z, w1, w2: np.sqrt(-0.5 * z ** 2) * w1 + np.cosh(z) * w2),
    ("abs(a(K,:)).^2.5 + real(a(K,:)).^2 - abs(a(K,:)).^-1",
     lambda z, w1, w2: abs(z) ** 2.5 + z.real ** 2 - abs(z) ** -1.0),
    ("(real(a(K,:)) < 0 | imag(a(K,:)) >= 0.5) + 2*(real(a(K,:)) > 0 & ~(imag(a(K,:)) > 0))",
     lambda z, w1, w2: ((z.real < 0) | (z.imag >= 0.5)) + 2.0 * ((z.real > 0) & ~(z.imag > 0))),
    ("tan(a(K,:)) + sin(a(K,:)).*cos(a(K,:)) + sinh(a(K,:))",
     lambda z, w1, w2: np.tan(z) + np.sin(z) * np.cos(z) + np.sinh(z)),
    ("exp(a(K,:)).*log(a(K,:))./sqrt(a(K,:))", lambda z, w1, w2: np.exp(z) * np.log(z) / np.sqrt(z)),
    ("1./a(K,:) - 2.\\a(K,:) + a(K,:)'", lambda z, w1, w2: 1 / z - z / 2 + np.conj(z)),
    ("(w(1,:) + 1i*w(2,:))/sqrt(2) - 0.25i*a(K,:).^2", lambda z, w1, w2: (w1 + 1j * w2) / np.sqrt(2) - 0.25j * z ** 2),
    ("sec(real(a(K,:))) + csc(imag(a(K,:))) + cot(a(K,:)) + csch(a(K,:))",
     lambda z, w1, w2: 1 / np.cos(z.real) + 1 / np.sin(z.imag) + 1 / np.tan(z) + 1 / np.sinh(z)),
]


def _cut(src, head):
    """The definition that starts with `head`, up to its closing brace at column 0."""
    i = src.index(head)
    j = src.index("\n}\n", i)
    return src[i:j + 3]


def _generated_source(tmp, deriv, fields):
    """The resident-path NVRTC source the library generates for a 0-D problem with this drift."""
    from xspde_matlab_b200 import _lib
    from xspde_matlab_b200.xsim import make_problem, xpreferences
    d = dict(dimensions=1, points=[5], ranges=[1.0], fields=fields, noises=2, precision="fp64",
             ensembles=[4, 1, 1], deriv=deriv, initial="@(v,p) zeros(%d,1)" % fields,
             observe=["@(a,p) real(a(1,:))"])
    old = os.environ.get("XSPDE_B200_DUMP"), os.environ.get("XSPDE_B200_CACHE")
    os.environ["XSPDE_B200_DUMP"] = str(tmp / "dump")
    os.environ["XSPDE_B200_CACHE"] = str(tmp / "cache")
    try:
        q = xpreferences([d])[0]
        pr, keep = make_problem(q)
        log = ctypes.create_string_buffer(1 << 16)
        _lib.check(_lib.lib().xs_compile_check(ctypes.byref(pr), log, len(log)))
    finally:
        for k, v in zip(("XSPDE_B200_DUMP", "XSPDE_B200_CACHE"), old):
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    srcs = [open(tmp / "dump" / f).read() for f in os.listdir(tmp / "dump") if f.startswith("xs_resident")]
    assert len(srcs) == 1
    return srcs[0]


def _build(tmp, code, name):
    cpp = tmp / (name + ".cpp")
    cpp.write_text(code)
    so = tmp / (name + ".so")
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-o", str(so), str(cpp)],
                   check=True, capture_output=True, text=True)
    return ctypes.CDLL(str(so))


GROUP = 11  # field components per generated problem (the library takes up to 16)


@pytest.fixture(scope="module")
def drift(tmp_path_factory):
    """One .so with eval_deriv<g>(n, a, w, out) for each group of CASES; each group is the
    drift [e1; e2; ...] of one problem, component k reading a(k,:)."""
    code = "#define XS_REAL double\n#define XS_FP64 1\n" + SHIM
    code += open(os.path.join(KERNELS, "xs_prelude.cuh")).read().replace("#pragma once", "")
    srcs = []
    for g in range(0, len(CASES), GROUP):
        part = CASES[g:g + GROUP]
        K = len(part)
        tmp = tmp_path_factory.mktemp("drift%d" % g)
        deriv = "@(a,w,p) [" + "; ".join(e.replace("K", str(k + 1)) for k, (e, _) in enumerate(part)) + "]"
        src = _generated_source(tmp, deriv, K)
        srcs.append(src)
        fn = _cut(src, "__device__ __forceinline__ void xs_deriv(")
        code += fn.replace("void xs_deriv(", "void xs_deriv_%d(" % g)
        code += r"""
extern "C" void eval_deriv_%(g)d(int n, const double* a, const double* w, double* out) {
  for (int i = 0; i < n; ++i) {
    cx av[%(K)d], o[%(K)d];
    real wv[2] = {w[2 * i], w[2 * i + 1]};
    for (int k = 0; k < %(K)d; ++k) av[k] = mkcx(a[2 * (i * %(K)d + k)], a[2 * (i * %(K)d + k) + 1]);
    xs_deriv_%(g)d(av, wv, nullptr, 0, 0, 0, 0, nullptr, nullptr, 0, 0, o);
    for (int k = 0; k < %(K)d; ++k) { out[2 * (i * %(K)d + k)] = o[k].re; out[2 * (i * %(K)d + k) + 1] = o[k].im; }
  }
}
""" % dict(K=K, g=g)
    L = _build(tmp_path_factory.mktemp("drift_so"), code, "drift")
    for g in range(0, len(CASES), GROUP):
        getattr(L, "eval_deriv_%d" % g).argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return L, "\n".join(srcs)


def test_generated_drift_follows_matlab_semantics(drift):
    L, _ = drift
    rng = np.random.default_rng(11)
    n = 400
    bad = []
    for g in range(0, len(CASES), GROUP):
        part = CASES[g:g + GROUP]
        K = len(part)
        z = (rng.standard_normal((n, K)) + 1j * rng.standard_normal((n, K))) * 1.3
        z[:8] = np.array([-2.5, -1.5, -0.5, 0.5, 1.5, 2.5, 3.5, -3.5])[:, None] + 1j * z[:8].imag  # exact halves
        w = rng.standard_normal((n, 2))
        a = np.ascontiguousarray(np.stack([z.real, z.imag], axis=-1))
        out = np.empty_like(a)
        getattr(L, "eval_deriv_%d" % g)(n, a.ctypes.data, np.ascontiguousarray(w).ctypes.data, out.ctypes.data)
        got = out[..., 0] + 1j * out[..., 1]
        for k, (expr, ref) in enumerate(part):
            want = np.asarray(ref(z[:, k], w[:, 0], w[:, 1]), dtype=complex) * np.ones(n)
            err = np.abs(got[:, k] - want) / np.maximum(1.0, np.abs(want))
            if not np.max(err) < 1e-12:
                bad.append("%s: max rel err %.2e" % (expr, np.max(err)))
    assert not bad, "\n".join(bad)


def test_real_arguments_leave_the_reals_where_matlab_does(drift):
    """sqrt/log/fractional power of a real expression are evaluated in complex arithmetic."""
    _, src = drift
    body = _cut(src, "__device__ __forceinline__ void xs_deriv(")  # the first group
    assert re.search(r"xs_sqrt\(mkcx\(", body) and re.search(r"xs_log\(mkcx\(", body)
    assert "xs_pow(" in body and "xs_powi<3>" in body and "xs_powi<-2>" in body


NOISE = r"""
template <int NC> void site(real* z, u32 s, u32 e, u32 q, u32 seq, u32 seed, u32 block) {
  xs_normals<NC>(z, s, e, q, seq, seed, block);
}
extern "C" void normals(int nc, unsigned s, unsigned e, unsigned q, unsigned seq, unsigned seed, unsigned block,
                        double* out) {
  real z[8];
  switch (nc) {
    case 1: site<1>(z, s, e, q, seq, seed, block); break;
    case 2: site<2>(z, s, e, q, seq, seed, block); break;
    case 3: site<3>(z, s, e, q, seq, seed, block); break;
    case 5: site<5>(z, s, e, q, seq, seed, block); break;
    default: return;
  }
  for (int c = 0; c < nc; ++c) out[c] = (double)z[c];
}
extern "C" void normals_paired(unsigned s, unsigned e, unsigned q, unsigned seq, unsigned seed, unsigned block,
                               double* out) {
  real z[2];
  xs_normals_site<2>(z, s, e, q, seq, seed, block);
  out[0] = (double)z[0];
  out[1] = (double)z[1];
}
extern "C" double knormal(int k, unsigned s, unsigned e, unsigned q, unsigned seq, unsigned seed, unsigned block) {
  return (double)xs_knormal(k, s, e, q, seq, seed, block);
}
"""


def _noise_lib(tmp, fp64):
    src = open(os.path.join(KERNELS, "xs_noise.cuh")).read()
    i = src.index("#define XS_PAIRED")
    j = src.index("\n}\n", src.index("void xs_normals_pair(")) + 3
    code = "#define XS_REAL %s\n#define XS_FP64 %d\n#define XS_ND 1\n#define XS_N1 16\n" % (
        "double" if fp64 else "float", int(fp64))
    code += SHIM + open(os.path.join(KERNELS, "xs_prelude.cuh")).read().replace("#pragma once", "")
    code += src[i:j] + NOISE
    L = _build(tmp, code, "noise%d" % int(fp64))
    L.normals.argtypes = [ctypes.c_int] + [ctypes.c_uint] * 6 + [ctypes.c_void_p]
    L.normals_paired.argtypes = [ctypes.c_uint] * 6 + [ctypes.c_void_p]
    L.knormal.argtypes = [ctypes.c_int] + [ctypes.c_uint] * 6
    L.knormal.restype = ctypes.c_double
    return L


@pytest.mark.parametrize("fp64,tol", [(True, 1e-13), (False, 2e-4)])
def test_kernel_noise_matches_oracle_stream(tmp_path, fp64, tol):
    """xs_normals (plain sites, 1-5 components), xs_normals_site (paired sites of a 16-point
    first dimension) and xs_knormal (k-space stream) against oracle/philox.py; FP32 within its
    Box-Muller rounding (the largest words give r = 0 where FP64 gives 1.5e-5)."""
    L = _noise_lib(tmp_path, fp64)
    seed, block, seq, draw = 7, 3, 1, 5
    nspace, nens = 48, 6
    out = np.empty(8)
    for nc in (1, 2, 3, 5):
        ref = philox.normals(nc, nspace, nens, draw, block, seed, seq)
        for s in range(0, nspace, 5):
            for e in range(nens):
                L.normals(nc, s, e, draw, seq, seed, block, out.ctypes.data)
                assert np.max(np.abs(out[:nc] - ref[:, s, e])) < tol * max(1.0, np.max(np.abs(ref[:, s, e])))
    ref = philox.normals(2, nspace, nens, draw, block, seed, seq, 16)
    for s in range(nspace):
        for e in range(0, nens, 2):
            L.normals_paired(s, e, draw, seq, seed, block, out.ctypes.data)
            assert np.max(np.abs(out[:2] - ref[:, s, e])) < tol * max(1.0, np.max(np.abs(ref[:, s, e])))
    ref = philox.normals(5, nspace, nens, draw, block, seed, seq, kstream=True)
    for k in range(5):
        for s in range(0, nspace, 7):
            got = L.knormal(k, s, 2, draw, seq, seed, block)
            assert abs(got - ref[k, s, 2]) < tol * max(1.0, abs(ref[k, s, 2]))


# Drifts of 2D periodic problems, which run on the streaming row pass.  There the midpoint
# update a0 + h D(a) is generated as c0 + h dep(a): c0 = a0 + h inv(w, x, y, t) holds the
# terms that do not read the field, formed once per site, and the iterations add the rest.
SPLIT = [
    ("-1i*(p.x.^2 + p.y.^2).*a + sin(p.t)*(w(1,:)+1i*w(2,:)) + 0.1i*a.*conj(a).*a + p.g*p.x",
     lambda a, w1, w2, x, y, t: -1j * (x ** 2 + y ** 2) * a + np.sin(t) * (w1 + 1j * w2) + 0.1j * a * np.conj(a) * a
     + 0.3 * x),
    ("exp(-p.t)*a - 0.3*cos(p.x).*w(1,:) + 1i*p.y",
     lambda a, w1, w2, x, y, t: np.exp(-t) * a - 0.3 * np.cos(x) * w1 + 1j * y),
    ("a.^2.*w(2,:) - conj(a).*w(1,:) + 0.2", lambda a, w1, w2, x, y, t: a ** 2 * w2 - np.conj(a) * w1 + 0.2),
    ("sqrt(abs(a)).*a + tanh(p.x - p.y).*w(1,:) - 0.5",
     lambda a, w1, w2, x, y, t: np.sqrt(abs(a)) * a + np.tanh(x - y) * w1 - 0.5),
    ("(1-abs(a).^2).*a - 0.5i*abs(a).^2.*a + 0.05*(w(1,:)+1i*w(2,:))/sqrt(2)",
     lambda a, w1, w2, x, y, t: (1 - abs(a) ** 2) * a - 0.5j * abs(a) ** 2 * a + 0.05 * (w1 + 1j * w2) / np.sqrt(2)),
    ("1i*p.g*(a - 1) + p.g^2*w(1,:).*w(2,:)",
     lambda a, w1, w2, x, y, t: 0.3j * (a - 1) + 0.09 * w1 * w2),
]


def _stream_source(tmp, deriv):
    """The 2D streaming NVRTC source the library generates for a 256 x 256 periodic problem."""
    from xspde_matlab_b200 import _lib
    from xspde_matlab_b200.xsim import make_problem, xpreferences
    d = dict(dimensions=3, points=[3, 256, 256], ranges=[1.0, 20.0, 20.0], steps=1, ensembles=[4, 1, 1], noises=2,
             method="MP", precision="fp64", params={"g": 0.3}, deriv=deriv, initial="@(v,p) 1 + 0*p.x",
             linear="@(p) 0.5i*(p.Dx.^2+p.Dy.^2)", observe=["@(a,p) abs(a).^2"])
    old = os.environ.get("XSPDE_B200_DUMP"), os.environ.get("XSPDE_B200_CACHE")
    os.environ["XSPDE_B200_DUMP"] = str(tmp / "dump")
    os.environ["XSPDE_B200_CACHE"] = str(tmp / "cache")
    try:
        q = xpreferences([d])[0]
        pr, keep = make_problem(q)
        log = ctypes.create_string_buffer(1 << 16)
        _lib.check(_lib.lib().xs_compile_check(ctypes.byref(pr), log, len(log)))
    finally:
        for k, v in zip(("XSPDE_B200_DUMP", "XSPDE_B200_CACHE"), old):
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    srcs = [open(tmp / "dump" / f).read() for f in os.listdir(tmp / "dump") if f.startswith("xs_stream")]
    assert len(srcs) == 1
    return srcs[0]


def test_streaming_drift_split_matches_unsplit_update(tmp_path):
    """For drifts with coordinates, time, named scalars, multiplicative and additive noise:
    the generated drift equals NumPy's evaluation, and c0 + h dep(a) equals a0 + h D(a)."""
    code = "#define XS_REAL double\n#define XS_FP64 1\n" + SHIM
    code += open(os.path.join(KERNELS, "xs_prelude.cuh")).read().replace("#pragma once", "")
    for k, (expr, _) in enumerate(SPLIT):
        src = _stream_source(tmp_path / ("s%d" % k), "@(a,w,p) " + expr)
        assert "#define XS_DSPLIT 1" in src, expr
        for name in ("xs_deriv", "xs_deriv_c0", "xs_deriv_step"):
            fn = _cut(src, "__device__ __forceinline__ void %s(" % name)
            fn = fn.replace("void %s(" % name, "void %s_%d(" % (name, k))
            code += fn
        code += r"""
extern "C" void update_%(k)d(int n, const double* a, const double* a0, const double* w, const double* xyt, double h,
                            double* out) {
  for (int i = 0; i < n; ++i) {
    cx av[1] = {mkcx(a[2 * i], a[2 * i + 1])}, a0v[1] = {mkcx(a0[2 * i], a0[2 * i + 1])}, d[1], c0[1], s[1];
    real wv[2] = {w[2 * i], w[2 * i + 1]};
    const real x = xyt[3 * i], y = xyt[3 * i + 1], t = xyt[3 * i + 2];
    xs_deriv_%(k)d(av, wv, nullptr, x, y, 0, t, nullptr, nullptr, 0, 0, d);
    xs_deriv_c0_%(k)d(av, a0v, h, wv, nullptr, x, y, 0, t, nullptr, nullptr, 0, 0, c0);
    xs_deriv_step_%(k)d(av, c0, h, wv, nullptr, x, y, 0, t, nullptr, nullptr, 0, 0, s);
    out[6 * i + 0] = d[0].re; out[6 * i + 1] = d[0].im;
    out[6 * i + 2] = a0v[0].re + h * d[0].re; out[6 * i + 3] = a0v[0].im + h * d[0].im;
    out[6 * i + 4] = s[0].re; out[6 * i + 5] = s[0].im;
  }
}
""" % dict(k=k)
    L = _build(tmp_path, code, "split")
    rng = np.random.default_rng(12)
    n = 300
    bad = []
    for k, (expr, ref) in enumerate(SPLIT):
        a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        a0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        w = rng.standard_normal((n, 2))
        xyt = np.stack([rng.uniform(-10, 10, n), rng.uniform(-10, 10, n), rng.uniform(0, 5, n)], axis=1)
        h = 0.013
        out = np.empty((n, 6))
        f = getattr(L, "update_%d" % k)
        f.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + [ctypes.c_double, ctypes.c_void_p]
        ai = np.ascontiguousarray(np.stack([a.real, a.imag], 1))
        a0i = np.ascontiguousarray(np.stack([a0.real, a0.imag], 1))
        f(n, ai.ctypes.data, a0i.ctypes.data, np.ascontiguousarray(w).ctypes.data, np.ascontiguousarray(xyt).ctypes.data,
          h, out.ctypes.data)
        d = out[:, 0] + 1j * out[:, 1]
        full = out[:, 2] + 1j * out[:, 3]
        split = out[:, 4] + 1j * out[:, 5]
        want = ref(a, w[:, 0], w[:, 1], xyt[:, 0], xyt[:, 1], xyt[:, 2])
        e1 = np.max(np.abs(d - want) / np.maximum(1.0, np.abs(want)))
        e2 = np.max(np.abs(split - full) / np.maximum(1.0, np.abs(full)))
        if not (e1 < 1e-12 and e2 < 1e-13):
            bad.append("%s: drift %.2e, split %.2e" % (expr, e1, e2))
    assert not bad, "\n".join(bad)
