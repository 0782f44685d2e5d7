// Ahead-of-time kernels (compiled by nvcc for sm_100a) that do not depend on
// the problem: layout conversion between the MATLAB host layout and the
// device layout.  Problem kernels are generated and compiled by NVRTC.
#include <cuda_runtime.h>

#include "xs_aot.hpp"

// [F, NS, E] (MATLAB, field fastest) <-> [E][F][NS] (device), complex FP64.
extern "C" __global__ void xs_aot_reorder(const double2* __restrict__ src, double2* __restrict__ dst, int F, int NS,
                                          long long E, int to_device) {
  const long long total = (long long)F * NS * E;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / ((long long)F * NS);
    const int r = (int)(i % ((long long)F * NS));
    const int f = r / NS, s = r % NS;
    const long long m = f + (long long)F * (s + (long long)NS * e);
    if (to_device) dst[i] = src[m];
    else dst[m] = src[i];
  }
}

extern "C" int xs_aot_reorder_launch(const void* src, void* dst, int F, int NS, long long E, int to_device,
                                      cudaStream_t st) {
  const long long total = (long long)F * NS * E;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  xs_aot_reorder<<<blocks, 256, 0, st>>>((const double2*)src, (double2*)dst, F, NS, E, to_device);
  return (int)cudaGetLastError();
}

// Block means into MATLAB's av{o}(lines, time, space) order, one block after
// another: output element (b, o, l, n, s) <- device [b][n][k], k the line's
// site row (site observables) or its scalar slot.  Writes are contiguous.
extern "C" __global__ void xs_aot_av_matlab(const double2* __restrict__ src, double2* __restrict__ dst, const XsAvMap m,
                                            int nblocks) {
  const long long total = (long long)nblocks * m.per_block;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / m.per_block, r = i % m.per_block;
    int o = 0;
    while (o + 1 < m.nobs && r >= m.o_off[o + 1]) ++o;
    const long long idx = r - m.o_off[o];
    const int l = (int)(idx % m.lines[o]);
    const long long q = idx / m.lines[o];
    const int n = (int)(q % m.npts);
    const long long s = q / m.npts;
    const long long k = m.spatial[o] ? (long long)(m.out_off[o] + l) * m.NS + s
                                     : (long long)m.nout_site * m.NS + m.out_off[o] + l;
    dst[i] = src[(b * m.npts + n) * m.stride + k];
  }
}

extern "C" int xs_aot_av_matlab_launch(const void* src, void* dst, const XsAvMap* m, int nblocks, cudaStream_t st) {
  const long long total = (long long)nblocks * m->per_block;
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  xs_aot_av_matlab<<<(unsigned)blocks, 256, 0, st>>>((const double2*)src, (double2*)dst, *m, nblocks);
  return (int)cudaGetLastError();
}

// Ensemble moments over blocks (Simulator/xensemble.m:98-101): with D_b the
// real part of block b's means, mom[k] (+)= scale * sum_b D_b[k] and
// mom[n + k] (+)= scale * sum_b D_b[k]^2, blocks summed in order with
// Neumaier compensation.  One thread per element; block reads are coalesced.
extern "C" __global__ void xs_aot_block_moments(const double2* __restrict__ av, long long n, int nblocks, double scale,
                                                double* __restrict__ mom, int accumulate) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    double s1 = 0, c1 = 0, s2 = 0, c2 = 0;
    for (int b = 0; b < nblocks; ++b) {
      const double d = av[(long long)b * n + k].x;
      double t = s1 + d;
      c1 += fabs(s1) >= fabs(d) ? (s1 - t) + d : (d - t) + s1;
      s1 = t;
      const double d2 = d * d;
      t = s2 + d2;
      c2 += fabs(s2) >= fabs(d2) ? (s2 - t) + d2 : (d2 - t) + s2;
      s2 = t;
    }
    const double m1 = (s1 + c1) * scale, m2 = (s2 + c2) * scale;
    if (accumulate) {
      mom[k] += m1;
      mom[n + k] += m2;
    } else {
      mom[k] = m1;
      mom[n + k] = m2;
    }
  }
}

extern "C" int xs_aot_block_moments_launch(const void* av, long long n, int nblocks, double scale, void* mom,
                                            int accumulate, cudaStream_t st) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  xs_aot_block_moments<<<(unsigned)blocks, 256, 0, st>>>((const double2*)av, n, nblocks, scale, (double*)mom,
                                                         accumulate);
  return (int)cudaGetLastError();
}
