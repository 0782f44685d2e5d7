// Device prelude for the xSPDE B200 kernels (compiled by NVRTC for sm_100a).
// The generated problem header defines XS_REAL and the problem constants
// before this file is included.
#pragma once

typedef XS_REAL real;
typedef unsigned int u32;
typedef unsigned long long u64;

#ifndef INFINITY
#define INFINITY __int_as_float(0x7f800000)
#endif
#ifndef NAN
#define NAN __int_as_float(0x7fffffff)
#endif

struct __align__(2 * sizeof(real)) cx {
  real re, im;
};

__device__ __forceinline__ cx mkcx(real r, real i) { cx z; z.re = r; z.im = i; return z; }
// a * b + c with one rounding
#if XS_FP64
__device__ __forceinline__ real xs_fma(real a, real b, real c) { return fma(a, b, c); }
#else
__device__ __forceinline__ real xs_fma(real a, real b, real c) { return fmaf(a, b, c); }
#endif
// a * b rounded on its own, never contracted into a following add.  The coarse
// pass's noise (w1 s + w2 s) / 2 then rounds both scaled draws first, as
// Simulator/xnoise.m:32-35 does, so it equals the mean of the fine pass's two
// scaled draws bit for bit (a quantity that is the same in both check passes
// then has a step error of exactly zero, as in the reference).
#if XS_FP64
__device__ __forceinline__ real xs_mul_rn(real a, real b) { return __dmul_rn(a, b); }
#else
__device__ __forceinline__ real xs_mul_rn(real a, real b) { return __fmul_rn(a, b); }
#endif
__device__ __forceinline__ cx operator+(cx a, cx b) { return mkcx(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ cx operator-(cx a, cx b) { return mkcx(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ cx operator-(cx a) { return mkcx(-a.re, -a.im); }
__device__ __forceinline__ cx operator*(cx a, cx b) {
  return mkcx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__device__ __forceinline__ cx operator*(real a, cx b) { return mkcx(a * b.re, a * b.im); }
__device__ __forceinline__ cx operator*(cx a, real b) { return mkcx(a.re * b, a.im * b); }
__device__ __forceinline__ cx operator+(real a, cx b) { return mkcx(a + b.re, b.im); }
__device__ __forceinline__ cx operator+(cx a, real b) { return mkcx(a.re + b, a.im); }
__device__ __forceinline__ cx operator-(real a, cx b) { return mkcx(a - b.re, -b.im); }
__device__ __forceinline__ cx operator-(cx a, real b) { return mkcx(a.re - b, a.im); }
__device__ __forceinline__ cx operator/(cx a, real b) { return mkcx(a.re / b, a.im / b); }
__device__ __forceinline__ cx operator/(cx a, cx b) {
  // Smith's algorithm (R. L. Smith, CACM 1962) to avoid overflow.
  if (fabs(b.re) >= fabs(b.im)) {
    real r = b.im / b.re, d = b.re + b.im * r;
    return mkcx((a.re + a.im * r) / d, (a.im - a.re * r) / d);
  } else {
    real r = b.re / b.im, d = b.re * r + b.im;
    return mkcx((a.re * r + a.im) / d, (a.im * r - a.re) / d);
  }
}
__device__ __forceinline__ cx operator/(real a, cx b) { return mkcx(a, (real)0) / b; }

// ---- elementary functions (real and complex overloads) ----------------------
__device__ __forceinline__ real xs_conj(real a) { return a; }
__device__ __forceinline__ cx xs_conj(cx a) { return mkcx(a.re, -a.im); }
__device__ __forceinline__ real xs_real(real a) { return a; }
__device__ __forceinline__ real xs_real(cx a) { return a.re; }
__device__ __forceinline__ real xs_imag(real) { return (real)0; }
__device__ __forceinline__ real xs_imag(cx a) { return a.im; }
__device__ __forceinline__ real xs_abs(real a) { return fabs(a); }
__device__ __forceinline__ real xs_abs(cx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ real xs_abs2(real a) { return a * a; }
__device__ __forceinline__ real xs_abs2(cx a) { return a.re * a.re + a.im * a.im; }
__device__ __forceinline__ real xs_angle(real a) { return a < 0 ? (real)3.14159265358979323846 : (real)0; }
__device__ __forceinline__ real xs_angle(cx a) { return atan2(a.im, a.re); }
__device__ __forceinline__ real xs_exp(real a) { return exp(a); }
__device__ __forceinline__ cx xs_exp(cx a) {
  real e = exp(a.re), s, c;
  sincos(a.im, &s, &c);
  return mkcx(e * c, e * s);
}
__device__ __forceinline__ cx xs_log(cx a) { return mkcx(log(hypot(a.re, a.im)), atan2(a.im, a.re)); }
__device__ __forceinline__ cx xs_sqrt(cx a) {
  // principal branch, as MATLAB's sqrt
  if (a.re == (real)0 && a.im == (real)0) return mkcx((real)0, a.im);
  real r = hypot(a.re, a.im);
  real s = sqrt((r + fabs(a.re)) * (real)0.5);
  if (a.re >= (real)0) return mkcx(s, a.im / (2 * s));
  return mkcx(fabs(a.im) / (2 * s), copysign(s, a.im));
}
__device__ __forceinline__ real xs_sin(real a) { return sin(a); }
__device__ __forceinline__ real xs_cos(real a) { return cos(a); }
__device__ __forceinline__ real xs_tan(real a) { return tan(a); }
__device__ __forceinline__ real xs_sinh(real a) { return sinh(a); }
__device__ __forceinline__ real xs_cosh(real a) { return cosh(a); }
__device__ __forceinline__ real xs_tanh(real a) { return tanh(a); }
__device__ __forceinline__ real xs_sech(real a) { return (real)1 / cosh(a); }
__device__ __forceinline__ real xs_csch(real a) { return (real)1 / sinh(a); }
__device__ __forceinline__ real xs_sec(real a) { return (real)1 / cos(a); }
__device__ __forceinline__ real xs_csc(real a) { return (real)1 / sin(a); }
__device__ __forceinline__ real xs_cot(real a) { return (real)1 / tan(a); }
__device__ __forceinline__ real xs_coth(real a) { return (real)1 / tanh(a); }
__device__ __forceinline__ real xs_atan(real a) { return atan(a); }
__device__ __forceinline__ real xs_sign(real a) { return a > 0 ? (real)1 : (a < 0 ? (real)-1 : (real)0); }
__device__ __forceinline__ real xs_floor(real a) { return floor(a); }
__device__ __forceinline__ real xs_ceil(real a) { return ceil(a); }
__device__ __forceinline__ real xs_round(real a) { return round(a); }
__device__ __forceinline__ real xs_fix(real a) { return trunc(a); }
__device__ __forceinline__ real xs_erf(real a) { return erf(a); }
__device__ __forceinline__ real xs_atan2(real a, real b) { return atan2(a, b); }
__device__ __forceinline__ real xs_min(real a, real b) { return fmin(a, b); }
__device__ __forceinline__ real xs_max(real a, real b) { return fmax(a, b); }
__device__ __forceinline__ real xs_mod(real a, real b) { return b == 0 ? a : a - floor(a / b) * b; }
__device__ __forceinline__ real xs_rem(real a, real b) { return b == 0 ? a : a - trunc(a / b) * b; }
__device__ __forceinline__ cx xs_sin(cx a) {
  real s, c;
  sincos(a.re, &s, &c);
  return mkcx(s * cosh(a.im), c * sinh(a.im));
}
__device__ __forceinline__ cx xs_cos(cx a) {
  real s, c;
  sincos(a.re, &s, &c);
  return mkcx(c * cosh(a.im), -s * sinh(a.im));
}
__device__ __forceinline__ cx xs_sinh(cx a) {
  real s, c;
  sincos(a.im, &s, &c);
  return mkcx(sinh(a.re) * c, cosh(a.re) * s);
}
__device__ __forceinline__ cx xs_cosh(cx a) {
  real s, c;
  sincos(a.im, &s, &c);
  return mkcx(cosh(a.re) * c, sinh(a.re) * s);
}
__device__ __forceinline__ cx xs_tan(cx a) { return xs_sin(a) / xs_cos(a); }
__device__ __forceinline__ cx xs_tanh(cx a) { return xs_sinh(a) / xs_cosh(a); }
__device__ __forceinline__ cx xs_sech(cx a) { return (real)1 / xs_cosh(a); }
__device__ __forceinline__ cx xs_csch(cx a) { return (real)1 / xs_sinh(a); }
__device__ __forceinline__ cx xs_sec(cx a) { return (real)1 / xs_cos(a); }
__device__ __forceinline__ cx xs_csc(cx a) { return (real)1 / xs_sin(a); }
__device__ __forceinline__ cx xs_cot(cx a) { return xs_cos(a) / xs_sin(a); }
__device__ __forceinline__ cx xs_coth(cx a) { return xs_cosh(a) / xs_sinh(a); }
__device__ __forceinline__ cx xs_sign(cx a) {
  real r = hypot(a.re, a.im);
  return r == 0 ? mkcx(0, 0) : mkcx(a.re / r, a.im / r);
}
__device__ __forceinline__ cx xs_asin(cx z) {  // -i log(iz + sqrt(1 - z^2))
  cx iz = mkcx(-z.im, z.re);
  cx w = xs_log(iz + xs_sqrt((real)1 - z * z));
  return mkcx(w.im, -w.re);
}
__device__ __forceinline__ cx xs_acos(cx z) {
  cx s = xs_asin(z);
  return mkcx((real)1.57079632679489661923 - s.re, -s.im);
}
__device__ __forceinline__ cx xs_atan(cx z) {  // (i/2) log((i+z)/(i-z))
  cx w = xs_log(mkcx(z.re, 1 + z.im) / mkcx(-z.re, 1 - z.im));
  return mkcx(-w.im * (real)0.5, w.re * (real)0.5);
}
__device__ __forceinline__ cx xs_floor(cx a) { return mkcx(floor(a.re), floor(a.im)); }
__device__ __forceinline__ cx xs_ceil(cx a) { return mkcx(ceil(a.re), ceil(a.im)); }
__device__ __forceinline__ cx xs_round(cx a) { return mkcx(round(a.re), round(a.im)); }
__device__ __forceinline__ cx xs_fix(cx a) { return mkcx(trunc(a.re), trunc(a.im)); }

template <int N> __device__ __forceinline__ real xs_powi(real a) {
  if (N == 0) return (real)1;
  if (N < 0) return (real)1 / xs_powi<(N < 0 ? -N : 1)>(a);
  real r = a;
#pragma unroll
  for (int i = 1; i < (N > 0 ? N : 1); ++i) r *= a;
  return r;
}
template <int N> __device__ __forceinline__ cx xs_powi(cx a) {
  if (N == 0) return mkcx((real)1, (real)0);
  if (N < 0) return (real)1 / xs_powi<(N < 0 ? -N : 1)>(a);
  cx r = a;
#pragma unroll
  for (int i = 1; i < (N > 0 ? N : 1); ++i) r = r * a;
  return r;
}
__device__ __forceinline__ cx xs_pow(cx a, cx b) {
  if (a.re == 0 && a.im == 0) return mkcx((real)0, (real)0);
  return xs_exp(b * xs_log(a));
}
__device__ __forceinline__ cx xs_pow(real a, cx b) { return xs_pow(mkcx(a, 0), b); }
__device__ __forceinline__ cx xs_pow(cx a, real b) { return xs_pow(a, mkcx(b, 0)); }
__device__ __forceinline__ cx xs_pow(real a, real b) {
  if (a >= 0) return mkcx(pow(a, b), (real)0);
  return xs_pow(mkcx(a, 0), mkcx(b, 0));
}
__device__ __forceinline__ real xs_lt(real a, real b) { return a < b ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_lt(cx a, real b) { return a.re < b ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_lt(real a, cx b) { return a < b.re ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_lt(cx a, cx b) { return a.re < b.re ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_le(real a, real b) { return a <= b ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_le(cx a, real b) { return a.re <= b ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_le(real a, cx b) { return a <= b.re ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_le(cx a, cx b) { return a.re <= b.re ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_eq(real a, real b) { return a == b ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_eq(cx a, real b) { return (a.re == b && a.im == 0) ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_eq(real a, cx b) { return xs_eq(b, a); }
__device__ __forceinline__ real xs_eq(cx a, cx b) { return (a.re == b.re && a.im == b.im) ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_nz(real a) { return a != 0 ? (real)1 : (real)0; }
__device__ __forceinline__ real xs_nz(cx a) { return (a.re != 0 || a.im != 0) ? (real)1 : (real)0; }
template <class A, class B> __device__ __forceinline__ real xs_and(A a, B b) { return xs_nz(a) * xs_nz(b); }
template <class A, class B> __device__ __forceinline__ real xs_or(A a, B b) {
  return (xs_nz(a) + xs_nz(b)) > 0 ? (real)1 : (real)0;
}
template <class A> __device__ __forceinline__ real xs_not(A a) { return (real)1 - xs_nz(a); }

// ---- Philox4x32-10 (Salmon et al., SC'11) and Box-Muller (1958) ------------
__device__ __forceinline__ uint4 xs_philox(uint4 c, u32 k0, u32 k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    // one widening 32 x 32 -> 64-bit multiply gives both halves of each product
    const unsigned long long p0 = (unsigned long long)c.x * 0xD2511F53u;
    const unsigned long long p1 = (unsigned long long)c.z * 0xCD9E8D57u;
    c = make_uint4((u32)(p1 >> 32) ^ c.y ^ k0, (u32)p1, (u32)(p0 >> 32) ^ c.w ^ k1, (u32)p0);
  }
  return c;
}

// Box-Muller pair from two 32-bit words, u = (x + 1/2) 2^-32.
__device__ __forceinline__ void xs_boxmuller(u32 x0, u32 x1, real& z0, real& z1) {
#if XS_FP64
  const double u0 = ((double)x0 + 0.5) * 2.3283064365386963e-10;
  const double u1 = ((double)x1 + 0.5) * 2.3283064365386963e-10;
  const double r = sqrt(-2.0 * log(u0));
  double s, c;
  sincospi(2.0 * u1, &s, &c);
  z0 = r * c;
  z1 = r * s;
#else
  // FP32 fields: hardware approximations (__logf, __sincosf).  The angle is
  // taken in (-pi, pi): cos(2 pi u) = -cos(2 pi (u - 1/2)), likewise sin.
  const float u0 = ((float)x0 + 0.5f) * 2.3283064365386963e-10f;
  const float hu = (float)((int)(x1 ^ 0x80000000u)) * 2.3283064365386963e-10f + 1.16415321826934814e-10f;
  // u0 rounds to 1 in FP32 for the largest words (q = 0): r = 0 there, as sqrtf gives
  const float q = -2.0f * __logf(u0);
  const float r = q > 0.0f ? q * rsqrtf(q) : 0.0f;
  float s, c;
  __sincosf(6.28318530717958648f * hu, &s, &c);
  z0 = -r * c;
  z1 = -r * s;
#endif
}

// NC normals for lattice site s, trajectory e (in its block), draw q.
template <int NC>
__device__ __forceinline__ void xs_normals(real* z, u32 s, u32 e, u32 q, u32 seq, u32 seed, u32 block) {
#pragma unroll
  for (int g = 0; g < (NC + 3) / 4; ++g) {
    const uint4 w = xs_philox(make_uint4(s, e, q, (u32)g | (seq << 16)), seed, block);
    real z0, z1, z2, z3;
    xs_boxmuller(w.x, w.y, z0, z1);
    if (4 * g + 0 < NC) z[4 * g + 0] = z0;
    if (4 * g + 1 < NC) z[4 * g + 1] = z1;
    if (4 * g + 2 < NC) {
      xs_boxmuller(w.z, w.w, z2, z3);
      z[4 * g + 2] = z2;
      if (4 * g + 3 < NC) z[4 * g + 3] = z3;
    }
  }
}

// One standard normal of component k from the k-space stream (k-filtered
// noises and randoms): the fourth counter word carries bit 15, no site pairing.
__device__ __forceinline__ real xs_knormal(int k, u32 s, u32 e, u32 q, u32 seq, u32 seed, u32 block) {
  const uint4 w = xs_philox(make_uint4(s, e, q, (u32)(k >> 2) | 0x8000u | (seq << 16)), seed, block);
  real z0, z1;
  if (k & 2) xs_boxmuller(w.z, w.w, z0, z1);
  else xs_boxmuller(w.x, w.y, z0, z1);
  return (k & 1) ? z1 : z0;
}

// Neumaier's compensated summation (A. Neumaier, ZAMM 54 (1974) 39-51) for the FP64
// moment sums: the running sum s and the correction c together hold the total to about
// one rounding of the exact sum, whatever the number of terms; the result is s + c.
__device__ __forceinline__ void xs_kadd(double& s, double& c, double x) {
  const double t = s + x;
  c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
  s = t;
}

// ---- block reductions --------------------------------------------------------
__device__ __forceinline__ double xs_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
