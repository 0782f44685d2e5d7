"""Generated device code checked on the CPU: the straight-line DFT-16 of the streaming FFTs
(butterflies with general twiddles folded into fused multiply-adds) against numpy's FFT, and
the MP drift split of the 256x256 GPE, c0 = a0 + h inv(w) then c0 + h dep(a), against
a0 + h D(a, w) of the unsplit drift (Applications/SDE/MP.m:16).  The functions are cut out
of the NVRTC source the library generates and compiled with g++ against small host
stand-ins for the complex type, in FP64."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

HOST = r"""
#include <cmath>
#define __device__
#define __forceinline__ inline
#define __restrict__
typedef double real;
struct cx { real re, im; };
inline cx mkcx(real r, real i) { cx z; z.re = r; z.im = i; return z; }
inline cx operator+(cx a, cx b) { return mkcx(a.re + b.re, a.im + b.im); }
inline cx operator-(cx a, cx b) { return mkcx(a.re - b.re, a.im - b.im); }
inline cx operator-(cx a) { return mkcx(-a.re, -a.im); }
inline cx operator*(cx a, cx b) { return mkcx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline cx operator*(real a, cx b) { return mkcx(a * b.re, a * b.im); }
inline cx operator*(cx a, real b) { return mkcx(a.re * b, a.im * b); }
inline cx operator+(real a, cx b) { return mkcx(a + b.re, b.im); }
inline cx operator+(cx a, real b) { return mkcx(a.re + b, a.im); }
inline cx operator-(real a, cx b) { return mkcx(a - b.re, -b.im); }
inline cx operator-(cx a, real b) { return mkcx(a.re - b, a.im); }
inline real xs_fma(real a, real b, real c) { return std::fma(a, b, c); }
inline real xs_abs2(real a) { return a * a; }
inline real xs_abs2(cx a) { return a.re * a.re + a.im * a.im; }
template <int R> void xs_dftR(cx (&v)[R]);
"""

WRAP = r"""
extern "C" void dft16(double* io) {
  cx v[16];
  for (int k = 0; k < 16; ++k) v[k] = mkcx(io[2 * k], io[2 * k + 1]);
  xs_dftR<16>(v);
  for (int k = 0; k < 16; ++k) { io[2 * k] = v[k].re; io[2 * k + 1] = v[k].im; }
}
// out[0..1] = a0 + h D(a, w); out[2..3] = c0 + h dep(a) with c0 = a0 + h inv(w)
extern "C" void mp_update(const double* a_, const double* a0_, const double* w, double h, double* out) {
  cx a[1] = {mkcx(a_[0], a_[1])}, a0[1] = {mkcx(a0_[0], a0_[1])}, d[1], c0[1], s[1];
  xs_deriv(a, w, nullptr, 0, 0, 0, 0, nullptr, nullptr, 0, 0, d);
  out[0] = a0[0].re + h * d[0].re;
  out[1] = a0[0].im + h * d[0].im;
  xs_deriv_c0(a, a0, h, w, nullptr, 0, 0, 0, 0, nullptr, nullptr, 0, 0, c0);
  xs_deriv_step(a, c0, h, w, nullptr, 0, 0, 0, 0, nullptr, nullptr, 0, 0, s);
  out[2] = s[0].re;
  out[3] = s[0].im;
}
"""


def _cut(src, head):
    """The definition that starts with `head`, up to its closing brace at column 0."""
    i = src.index(head)
    j = src.index("\n}\n", i)
    return src[i:j + 3]


@pytest.fixture(scope="module")
def generated(tmp_path_factory):
    from xspde_matlab_b200 import problems
    d = tmp_path_factory.mktemp("gen")
    old = os.environ.get("XSPDE_B200_DUMP"), os.environ.get("XSPDE_B200_CACHE")
    os.environ["XSPDE_B200_DUMP"] = str(d / "dump")
    os.environ["XSPDE_B200_CACHE"] = str(d / "cache")
    try:
        problems.compile_check("gpe_2d", precision="fp64")
    finally:
        for k, v in zip(("XSPDE_B200_DUMP", "XSPDE_B200_CACHE"), old):
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    srcs = [open(d / "dump" / f).read() for f in os.listdir(d / "dump") if f.startswith("xs_stream")]
    assert len(srcs) == 1
    src = srcs[0]
    assert "#define XS_DSPLIT 1" in src
    code = HOST
    code += _cut(src, "template <> __device__ __forceinline__ void xs_dftR<16>(cx (&v)[16]) {")
    for name in ("xs_deriv(", "xs_deriv_c0(", "xs_deriv_step("):
        code += _cut(src, "__device__ __forceinline__ void " + name)
    code += WRAP
    cpp = d / "gen.cpp"
    cpp.write_text(code)
    so = d / "gen.so"
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-o", str(so), str(cpp)],
                   check=True)
    L = ctypes.CDLL(str(so))
    L.dft16.argtypes = [ctypes.c_void_p]
    L.mp_update.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    return L, src


def test_generated_dft16_matches_numpy_fft(generated):
    L, src = generated
    assert re.search(r"xs_fma\(\(real\)[-0-9.e]+, q\d+\.im, q\d+\.re\)", src)  # folded butterflies are emitted
    rng = np.random.default_rng(5)
    for _ in range(20):
        x = rng.standard_normal(16) + 1j * rng.standard_normal(16)
        io = np.empty(32)
        io[0::2], io[1::2] = x.real, x.imag
        L.dft16(io.ctypes.data)
        got = io[0::2] + 1j * io[1::2]
        ref = np.fft.fft(x)
        assert np.max(np.abs(got - ref)) < 1e-13 * np.max(np.abs(ref))


def test_generated_drift_split_matches_unsplit_update(generated):
    L, _ = generated
    rng = np.random.default_rng(6)
    for _ in range(50):
        a = rng.standard_normal(2) * 1.5
        a0 = rng.standard_normal(2)
        w = rng.standard_normal(2)
        h = float(rng.uniform(0.001, 0.1))
        out = np.empty(4)
        L.mp_update(a.ctypes.data, a0.ctypes.data, w.ctypes.data, h, out.ctypes.data)
        ref = out[0] + 1j * out[1]
        assert abs((out[2] + 1j * out[3]) - ref) < 1e-14 * max(1.0, abs(ref))
        # and the unsplit update itself is the GPE drift (1 - |a|^2) a - 0.5i |a|^2 a + 0.05 xi
        az, a0z = a[0] + 1j * a[1], a0[0] + 1j * a0[1]
        n = abs(az) ** 2
        d = (1 - n) * az - 0.5j * n * az + 0.05 * (w[0] + 1j * w[1]) / np.sqrt(2)
        assert abs(ref - (a0z + h * d)) < 1e-14 * max(1.0, abs(ref))
