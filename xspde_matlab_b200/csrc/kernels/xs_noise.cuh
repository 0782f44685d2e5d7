// Noise mapping shared by the resident and streaming kernels (included after
// the problem constants).  Site pairing: with at most two components and an
// even number N1 of points along x, one Philox call serves sites i1 and
// i1 + N1/2 of the same x line: counter p = (i1 mod N1/2) + (N1/2)(s div N1),
// words (0,1) for the lower site and (2,3) for the upper one.  Otherwise each
// site has its own calls (xs_normals).  The CPU oracle uses the same rule.
#pragma once

#define XS_PAIRED(NC) ((NC) <= 2 && XS_ND >= 1 && XS_N1 > 1 && (XS_N1 % 2) == 0)

template <int NC>
__device__ __forceinline__ void xs_normals_site(real* z, u32 s, u32 e, u32 q, u32 seq, u32 seed, u32 block) {
  if (XS_PAIRED(NC)) {
    const u32 h = (u32)(XS_N1 / 2);
    const u32 i1 = s % (u32)XS_N1;
    const u32 p = i1 % h + h * (s / (u32)XS_N1);
    const uint4 w = xs_philox(make_uint4(p, e, q, seq << 16), seed, block);
    real z0, z1;
    if (i1 >= h) xs_boxmuller(w.z, w.w, z0, z1);
    else xs_boxmuller(w.x, w.y, z0, z1);
    z[0] = z0;
    if (NC > 1) z[NC > 1 ? 1 : 0] = z1;
  } else {
    xs_normals<NC>(z, s, e, q, seq, seed, block);
  }
}

// Both sites of pair p: zlo for i1 = p mod (N1/2) and zhi for i1 + N1/2.
template <int NC>
__device__ __forceinline__ void xs_normals_pair(real* zlo, real* zhi, u32 p, u32 e, u32 q, u32 seq, u32 seed,
                                                u32 block) {
  const uint4 w = xs_philox(make_uint4(p, e, q, seq << 16), seed, block);
  real a0, a1, b0, b1;
  xs_boxmuller(w.x, w.y, a0, a1);
  zlo[0] = a0;
  if (NC > 1) zlo[NC > 1 ? 1 : 0] = a1;
  xs_boxmuller(w.z, w.w, b0, b1);
  zhi[0] = b0;
  if (NC > 1) zhi[NC > 1 ? 1 : 0] = b1;
}

// p.noisegen / p.randomgen export (Simulator/xnoise.m:29-32, xrandom.m:20-23):
// out[c + NC (s + NS e)] = z_c(s, e) * scale for one block and draw, in the
// MATLAB layout [components, space, ens1].
template <int NC>
__device__ __forceinline__ void xs_export_normals(double* __restrict__ out, int ens1, u32 block, u32 draw, u32 seq,
                                                  u32 seed, double scale) {
  const size_t total = (size_t)XS_NS * (size_t)ens1;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const u32 s = (u32)(i % XS_NS), e = (u32)(i / XS_NS);
    real z[NC > 0 ? NC : 1];
    xs_normals_site<NC>(z, s, e, draw, seq, seed, block);
#pragma unroll
    for (int c = 0; c < NC; ++c) out[(size_t)c + (size_t)NC * i] = (double)z[c] * scale;
  }
}
extern "C" __global__ void xs_export_noise(double* out, int ens1, u32 block, u32 draw, u32 seq, u32 seed,
                                           double scale) {
#if XS_NW > 0
  xs_export_normals<XS_NW>(out, ens1, block, draw, seq, seed, scale);
#endif
}
extern "C" __global__ void xs_export_random(double* out, int ens1, u32 block, u32 draw, u32 seq, u32 seed,
                                            double scale) {
#if XS_NV > 0
  xs_export_normals<XS_NV>(out, ens1, block, draw, seq, seed, scale);
#endif
}

// Coarse space-time projections of the Wiener increments, the inputs of the
// learned control variate: for trajectory e and window tw,
//   out[e][((c*NT + tw)*NBY + by)*NBX + bx] =
//     sum over draws d0 + tw*DW .. d0 + (tw+1)*DW - 1 and over the sites of
//     lattice block (bx, by) of the standard normal z_c(site, e, draw)
//     weighted by exp(-decay (last draw of the window - draw)),
//   divided by sqrt(sum of squared weights * BW * BH) so that every feature
//   is N(0, 1) and the features of one trajectory are independent.  The lattice block (bx, by)
//   covers x indices i1lo + bx*BW .. + BW - 1 and y indices i2lo + by*BH ...
//   One CTA per (trajectory, window).
struct XsFeatArgs {
  int ntraj, ens1, block0, seq;
  u32 seed;
  int i1lo, i2lo, bw, bh, nbx, nby;
  int d0, dw, nt;
  float decay;  // draws weighted by exp(-decay * (last draw of the window - draw))
  float* out;
  int* status;
};

extern "C" __global__ void __launch_bounds__(256) xs_noise_features(const XsFeatArgs F) {
#if XS_NW > 0
  __shared__ float acc[XS_NW * 16 * 16];
  const int e = blockIdx.x / F.nt, tw = blockIdx.x % F.nt;
  if (e >= F.ntraj || F.nbx * F.nby > 256 || F.nbx < 1 || F.nby < 1) {
    if (threadIdx.x == 0) atomicOr(F.status, 2);
    return;
  }
  const int nb = F.nbx * F.nby;
  for (int i = threadIdx.x; i < XS_NW * nb; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  const int W = F.nbx * F.bw, H = F.nby * F.bh;
  const u32 blk = (u32)(F.block0 + e / F.ens1), el = (u32)(e % F.ens1);
  float wsum2 = 0.f;
  for (int q = 0; q < F.dw; ++q) {
    const u32 draw = (u32)(F.d0 + tw * F.dw + q);
    const float wq = __expf(-F.decay * (float)(F.dw - 1 - q));
    wsum2 += wq * wq;
    for (int i = threadIdx.x; i < W * H; i += blockDim.x) {
      const int lx = i % W, ly = i / W;
      const int i1 = F.i1lo + lx, i2 = F.i2lo + ly;
      const u32 s = (u32)(i2 * XS_N1 + i1);
      real z[XS_NW];
      xs_normals_site<XS_NW>(z, s, el, draw, (u32)F.seq, F.seed, blk);
      const int b = (ly / F.bh) * F.nbx + (lx / F.bw);
#pragma unroll
      for (int c = 0; c < XS_NW; ++c) atomicAdd(&acc[c * nb + b], wq * (float)z[c]);
    }
  }
  __syncthreads();
  const float sc = rsqrtf(wsum2 * (float)(F.bw * F.bh));
  for (int i = threadIdx.x; i < XS_NW * nb; i += blockDim.x) {
    const int c = i / nb, b = i % nb;
    F.out[(size_t)e * (XS_NW * F.nt * nb) + ((size_t)c * F.nt + tw) * nb + b] = acc[i] * sc;
  }
#endif
}
