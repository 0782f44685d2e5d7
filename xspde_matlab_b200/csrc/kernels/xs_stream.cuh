// Streaming-path kernels for 2D lattices whose field does not fit one CTA
// (Simulator/xpath.m:29-86 with Applications/SDE/MP.m and the periodic
// branch of Applications/SPDE/xprop.m / xtransform.m:45,60).
//
// Field layout in HBM: F[e][f][y][x], x fastest, complex `real`.  Between
// passes the field is held with the x direction Fourier transformed
// ("K state": kx, y).  One MP step (merged with its neighbour's half step):
//   xs_s_pass   column pass: FFT_y, multiply by exp(L dtr/2)^m (FP64 table,
//               m = 2 merges the previous step's second half with this step's
//               first half), IFFT_y
//   xs_x_nl     row pass: IFFT_x, midpoint iterations with the drift and
//               Philox noise generated in registers, 2a - a0, FFT_x
// Each pass reads and writes the field once: 4 N F s bytes per
// trajectory-step.  Observables (xs_x_obs) read the field once per output
// time and reduce over the trajectories of each block in a fixed order.
//
// 1D FFTs of length NX = RX*RX (and NY = RY*RY) use the four-step split:
// thread t of a line holds elements t + R*j (j < R) in registers; DFT-R over
// registers, twiddle W_N^(t k1), transpose through shared memory, DFT-R.
// The output lands in the same thread/element layout (index t + R*k2).
#pragma once

// XsStreamArgs, xs_dsmem, xs_smem_ok and xs_scalar_body: xs_stream_common.cuh

#define XS_RX XS_FFT_RX
#define XS_RY XS_FFT_RY
#define XS_NX XS_N1
#define XS_NY XS_N2
#define XS_XROWS (256 / XS_RX)          // rows per CTA in the row passes
#define XS_TX (256 / XS_RY)             // columns per CTA in the column pass
#define XS_OROWS XS_OBS_ROWS            // rows per CTA in the observation pass
#define XS_NRG (XS_NY / XS_OROWS)       // row groups per trajectory

template <int R> __device__ __forceinline__ void xs_dftR(cx (&v)[R]);

__device__ __forceinline__ cx xs_cj(cx a) { return mkcx(a.re, -a.im); }

// W_N^(t*k) for the four-step split, N = R*R: tw[k*R + t] = exp(-2 pi i t k / N)
// (t fastest, so the threads of a line read consecutive words), copied from
// the host-built table (L2-resident) into the CTA's shared memory, followed by
// the same table divided by N for the inverse transforms (N a power of two, so
// the division is exact).  XS_TWN(R) elements in all.
#define XS_TWN(R) (2 * (R) * (R))
template <int R, bool SCALED = true>
__device__ __forceinline__ void xs_fill_twiddles(cx* tw, const cx* __restrict__ src, int tid = -1, int nthr = 0) {
  if (tid < 0) {
    tid = threadIdx.x;
    nthr = blockDim.x;
  }
  const real sc = (real)(1.0 / (double)(R * R));
  for (int i = tid; i < R * R; i += nthr) {
    const cx w = src[i];
    tw[i] = w;
    if (SCALED) tw[R * R + i] = mkcx(w.re * sc, w.im * sc);
  }
}

// Forward DFT of N = R*R points held four-step style: thread t holds v[j] =
// x[t + R*j].  `buf` is the line's shared-memory scratch: element (k, t) of
// the R x R transpose lives at buf[(k*R + t)*LS] + padding chosen by the
// caller through LS (line stride between interleaved lines) and PAD; `sync`
// is the barrier that covers the threads of the line.  On return v[k2] =
// X[t + R*k2].
template <int R, int LS, int PAD, class Sync>
__device__ __forceinline__ void xs_fft4(cx (&v)[R], int t, const cx* __restrict__ tw, cx* buf, Sync sync) {
  xs_dftR<R>(v);  // v[k1] = sum_j x[t + R j] W_R^(j k1)
#pragma unroll
  for (int k = 1; k < R; ++k) v[k] = v[k] * tw[k * R + t];
#pragma unroll
  for (int k = 0; k < R; ++k) buf[(k * (R + PAD) + t) * LS] = v[k];
  sync();
#pragma unroll
  for (int n = 0; n < R; ++n) v[n] = buf[(t * (R + PAD) + n) * LS];
  sync();
  xs_dftR<R>(v);
}

// Inverse DFT (exp(+2 pi i n k / N) / N) in the same layout: conj, forward, conj.  The 1/N
// rides on the twiddle multiply (the second half of the table holds W/N; element k = 0, whose
// twiddle is 1, is scaled on its own): N is a power of two, so the result is bit-identical to
// scaling the output.
template <int R, int LS, int PAD, class Sync>
__device__ __forceinline__ void xs_ifft4(cx (&v)[R], int t, const cx* __restrict__ tw, cx* buf, Sync sync) {
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = xs_cj(v[k]);
  xs_dftR<R>(v);
  const real sc = (real)(1.0 / (double)(R * R));
  v[0] = mkcx(v[0].re * sc, v[0].im * sc);
  const cx* tws = tw + R * R;
#pragma unroll
  for (int k = 1; k < R; ++k) v[k] = v[k] * tws[k * R + t];
#pragma unroll
  for (int k = 0; k < R; ++k) buf[(k * (R + PAD) + t) * LS] = v[k];
  sync();
#pragma unroll
  for (int n = 0; n < R; ++n) v[n] = buf[(t * (R + PAD) + n) * LS];
  sync();
  xs_dftR<R>(v);
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = xs_cj(v[k]);
}

// Unnormalised inverse DFT (exp(+2 pi i n k / N), no 1/N): conj, forward, conj.  For callers that
// fold the 1/N into a multiply of their own.
template <int R, int LS, int PAD, class Sync>
__device__ __forceinline__ void xs_ifft4u(cx (&v)[R], int t, const cx* __restrict__ tw, cx* buf, Sync sync) {
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = xs_cj(v[k]);
  xs_fft4<R, LS, PAD>(v, t, tw, buf, sync);
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = xs_cj(v[k]);
}

struct XsWarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct XsBlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};


// ---- row passes -------------------------------------------------------------
// Shared memory: twiddles (RX*RX) + per-row transpose scratch (RX*(RX+1)).
#define XS_XLINE (XS_F * XS_RX * XS_RX > XS_RX * (XS_RX + 1) ? XS_F * XS_RX * XS_RX : XS_RX * (XS_RX + 1))
#define XS_XSMEM (XS_TWN(XS_RX) + XS_XROWS * XS_XLINE)

__device__ __forceinline__ void xs_row_coords(int y, int t, int j, real& x, real& yy) {
  x = (real)(XS_O1 + XS_DX1 * (double)(t + XS_RX * j));
  yy = (real)(XS_O2 + XS_DX2 * (double)y);
}

// XS_ROW_STAGE 1: the MP row pass stages its elements in shared memory so that the
// per-element drift/noise loop stays rolled (one copy of the code); 0 unrolls it over the
// registers, without the four shared-memory accesses per site: 4% faster in FP32 (1.437 against
// 1.499 ms per launch at 4096 trajectories of 256^2); FP64 keeps the stage (128 registers).
#ifndef XS_ROW_STAGE
#define XS_ROW_STAGE (XS_FP64 ? 1 : 0)
#endif

// MODE 0: initial field (expression or a_in) -> K state
// MODE 1: one MP step in x space (K state in, K state out)
// MODE 3: K state -> x-space a_out (FP64)
// Row block `cta` (XS_XROWS rows) by 256 threads tid = 0..255 with the shared
// memory `smem` (XS_XSMEM elements) and the barrier `bsync` of those threads.
template <int MODE, class Sync>
__device__ __forceinline__ void xs_xpass_core(const XsStreamArgs& A, int tid, size_t cta, cx* smem, Sync bsync) {
  cx* tw = smem;
  xs_fill_twiddles<XS_RX>(tw, A.tw_x, tid, 256);
  bsync();
  const int r = tid / XS_RX, t = tid % XS_RX;
  cx* buf = tw + XS_TWN(XS_RX) + r * XS_XLINE;
  const size_t row = cta * XS_XROWS + r;  // over ntraj * NY
  // XS_XROWS divides NY, so a CTA's rows share one trajectory: taking e from the CTA index lets
  // the compiler keep the trajectory, its block and the Philox keys warp-uniform
  const int e = (int)((cta * XS_XROWS) / XS_NY), y = (int)(row % XS_NY);
  const u32 blk = (u32)(A.block0 + e / A.ens1), el = (u32)(e % A.ens1);
  cx v[XS_F][XS_RX];
  cx* base = A.field + ((size_t)e * XS_F) * XS_NS + (size_t)y * XS_NX + t;
  XsWarpSync ws;
  if (MODE == 0) {
#pragma unroll
    for (int j = 0; j < XS_RX; ++j) {
      real x, yy;
      xs_row_coords(y, t, j, x, yy);
      const int s = y * XS_NX + t + XS_RX * j;
      cx a[XS_F];
      if (A.a_in) {
#pragma unroll
        for (int f = 0; f < XS_F; ++f) {
          const double2 q = A.a_in[((size_t)e * XS_F + f) * XS_NS + s];
          a[f] = mkcx((real)q.x, (real)q.y);
        }
      } else {
        real vv[XS_NV > 0 ? XS_NV : 1];
#if XS_NV > 0
        xs_normals_site<XS_NV>(vv, (u32)s, el, 0u, (u32)A.seq, A.seed, blk);
#pragma unroll
        for (int c = 0; c < XS_NV; ++c) vv[c] *= (real)A.vscale;
#endif
        xs_initial(vv, (const cx*)nullptr, x, yy, (real)0, A.params, a);
      }
#pragma unroll
      for (int f = 0; f < XS_F; ++f) v[f][j] = a[f];
    }
  } else {
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) v[f][j] = base[(size_t)f * XS_NS + XS_RX * j];
#pragma unroll
    for (int f = 0; f < XS_F; ++f) xs_ifft4<XS_RX, 1, 1>(v[f], t, tw, buf, ws);
  }
  if (MODE == 1) {
    // MP midpoint iterations (Applications/SDE/MP.m:13-23) at t + dtr/2.  The
    // row is staged in this row's shared scratch so that the per-element loop
    // stays rolled (one copy of the drift/noise code): each thread touches
    // only its own elements, stage[(f*RX + j)*RX + t].
    const real h = (real)(A.dtr * 0.5);
    const real tm = (real)(A.t + A.dtr * 0.5);
    // XS_ROW_STAGE 0: the per-element loop fully unrolled over the registers instead (no stage)
#if XS_ROW_STAGE
    cx* stage = buf;
#define XS_ROWEL(f, j) stage[((f) * XS_RX + (j)) * XS_RX + t]
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) stage[(f * XS_RX + j) * XS_RX + t] = v[f][j];
#else
#define XS_ROWEL(f, j) v[f][j]
#endif
    // One element: noise w (already scaled and, on a coarse pass, averaged),
    // midpoint iterations, 2a - a0.
    auto nl_element = [&](int j, const real* w) {
      real x, yy;
      xs_row_coords(y, t, j, x, yy);
      cx a0[XS_F], a[XS_F], d[XS_F];
#pragma unroll
      for (int f = 0; f < XS_F; ++f) a0[f] = a[f] = XS_ROWEL(f, j);
#if XS_DSPLIT
      // a = (a0 + h inv) + h dep(a): the drift's field-independent terms once per site
      cx c0[XS_F];
      xs_deriv_c0(a, a0, h, w, (const cx*)nullptr, x, yy, (real)0, tm, A.params, (const cx*)nullptr, 0, 0, c0);
#pragma unroll
      for (int it = 0; it < XS_ITER; ++it) {
        xs_deriv_step(a, c0, h, w, (const cx*)nullptr, x, yy, (real)0, tm, A.params, (const cx*)nullptr, 0, 0, d);
#pragma unroll
        for (int f = 0; f < XS_F; ++f) a[f] = d[f];
      }
#else
#pragma unroll
      for (int it = 0; it < XS_ITER; ++it) {
        xs_deriv(a, w, (const cx*)nullptr, x, yy, (real)0, tm, A.params, (const cx*)nullptr, 0, 0, d);
#pragma unroll
        for (int f = 0; f < XS_F; ++f) a[f] = a0[f] + h * d[f];
      }
#endif
#pragma unroll
      for (int f = 0; f < XS_F; ++f) XS_ROWEL(f, j) = (real)2 * a[f] - a0[f];
    };
    const real ws = (real)A.wscale;
#if XS_NW > 0 && XS_PAIRED(XS_NW)
    // one Philox call per pair of sites (x, x + NX/2) = elements (j, j + RX/2)
#if XS_ROW_STAGE
#pragma unroll 1
#else
#pragma unroll
#endif
    for (int j = 0; j < XS_RX / 2; ++j) {
      const u32 pidx = (u32)(t + XS_RX * j) + (u32)(XS_NX / 2) * (u32)y;
      real wl[XS_NW], wh[XS_NW];
      xs_normals_pair<XS_NW>(wl, wh, pidx, el, (u32)A.draw0, (u32)A.seq, A.seed, blk);
      if (A.draw1 >= 0) {
        real wl2[XS_NW], wh2[XS_NW];
        xs_normals_pair<XS_NW>(wl2, wh2, pidx, el, (u32)A.draw1, (u32)A.seq, A.seed, blk);
#pragma unroll
        for (int c = 0; c < XS_NW; ++c) {
          wl[c] = (xs_mul_rn(wl[c], ws) + xs_mul_rn(wl2[c], ws)) * (real)0.5;
          wh[c] = (xs_mul_rn(wh[c], ws) + xs_mul_rn(wh2[c], ws)) * (real)0.5;
        }
      } else {
#pragma unroll
        for (int c = 0; c < XS_NW; ++c) {
          wl[c] *= ws;
          wh[c] *= ws;
        }
      }
      nl_element(j, wl);
      nl_element(j + XS_RX / 2, wh);
    }
#else
#if XS_ROW_STAGE
#pragma unroll 1
#else
#pragma unroll
#endif
    for (int j = 0; j < XS_RX; ++j) {
      const u32 s = (u32)(y * XS_NX + t + XS_RX * j);
      real w[XS_NW > 0 ? XS_NW : 1];
#if XS_NW > 0
      xs_normals_site<XS_NW>(w, s, el, (u32)A.draw0, (u32)A.seq, A.seed, blk);
      if (A.draw1 >= 0) {
        real w2[XS_NW];
        xs_normals_site<XS_NW>(w2, s, el, (u32)A.draw1, (u32)A.seq, A.seed, blk);
#pragma unroll
        for (int c = 0; c < XS_NW; ++c) w[c] = (xs_mul_rn(w[c], ws) + xs_mul_rn(w2[c], ws)) * (real)0.5;
      } else {
#pragma unroll
        for (int c = 0; c < XS_NW; ++c) w[c] = w[c] * ws;
      }
#endif
      nl_element(j, w);
    }
#endif
#if XS_ROW_STAGE
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) v[f][j] = stage[(f * XS_RX + j) * XS_RX + t];
    __syncwarp();  // the FFT below reuses the scratch other threads may still read
#endif
#undef XS_ROWEL
  }
  if (MODE == 3) {
    bool bad = false;
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) {
        const cx q = v[f][j];
        if (!isfinite((double)q.re) || !isfinite((double)q.im)) bad = true;
        if (A.a_out)
          A.a_out[((size_t)e * XS_F + f) * XS_NS + (size_t)y * XS_NX + t + XS_RX * j] =
              make_double2((double)q.re, (double)q.im);
      }
    if (bad) atomicOr(A.status, 1);
    return;
  }
#pragma unroll
  for (int f = 0; f < XS_F; ++f) xs_fft4<XS_RX, 1, 1>(v[f], t, tw, buf, ws);
#pragma unroll
  for (int f = 0; f < XS_F; ++f)
#pragma unroll
    for (int j = 0; j < XS_RX; ++j) base[(size_t)f * XS_NS + XS_RX * j] = v[f][j];
}

template <int MODE>
__device__ __forceinline__ void xs_xpass_body(const XsStreamArgs& A) {
  // The grid covers ntraj*NY rows exactly; a CTA outside it leaves as a whole.
  if ((size_t)(blockIdx.x + 1) * XS_XROWS > (size_t)A.ntraj * XS_NY) {
    if (threadIdx.x == 0) atomicOr(A.status, 2);
    return;
  }
  if (!xs_smem_ok(XS_XSMEM * sizeof(cx), A.status)) return;
  xs_xpass_core<MODE>(A, threadIdx.x, blockIdx.x, (cx*)xs_dsmem, XsBlockSync());
}

// Minimum resident CTAs per SM of the MP row pass (register budget: 64 in FP32, 128 in FP64).
#ifndef XS_XPASS_MINB
#define XS_XPASS_MINB (XS_FP64 ? 2 : 4)
#endif
extern "C" __global__ void __launch_bounds__(256) xs_x_init(const XsStreamArgs A) { xs_xpass_body<0>(A); }
extern "C" __global__ void __launch_bounds__(256, XS_XPASS_MINB) xs_x_nl(const XsStreamArgs A) { xs_xpass_body<1>(A); }
extern "C" __global__ void __launch_bounds__(256) xs_x_final(const XsStreamArgs A) { xs_xpass_body<3>(A); }

// ---- RK4 row passes ------------------------------------------------------------
// Interaction-picture RK4 (Applications/SDE/RK4.m:7-42) with dt = dtr/2 and P the
// half-step propagator exp(L dtr/2) (applied by column passes on the field it
// acts on), one noise w for every stage of a step:
//   pass 1 (MODE 4):  a1 = a + dt D(a, t)                          -> field2
//   column passes:    a1 = P a1, a = P a
//   pass 2 (MODE 5):  a2 = a + dt D(a1, t + dt), a3 = a + 2 dt D(a2, t + dt),
//                     a = (a1 + 2 a2 + a3 - a)/3 -> field, a3 -> field2
//   column passes:    a = P a, a3 = P a3
//   pass 3 (MODE 6):  a = a + dt/3 D(a3, t + 2 dt)                 -> field
//                     (fuse: and the next step's pass 1 at the same time)
// Both fields stay in the K state between passes; pass 1 reads a but does not
// write it back.  Per step: 16 N F s bytes (four passes over two fields).
// Shared memory per row: two stages of XS_XLINE elements (field, field2), each
// also the transpose scratch of its field's transforms.
#define XS_XSMEM_RK (XS_TWN(XS_RX) + 2 * XS_XROWS * XS_XLINE)

template <int MODE>
__device__ __forceinline__ void xs_rk4_row(const XsStreamArgs& A) {
  if ((size_t)(blockIdx.x + 1) * XS_XROWS > (size_t)A.ntraj * XS_NY || blockDim.x != 256) {
    if (threadIdx.x == 0) atomicOr(A.status, 2);
    return;
  }
  if (!xs_smem_ok(XS_XSMEM_RK * sizeof(cx), A.status)) return;
  cx* tw = (cx*)xs_dsmem;
  xs_fill_twiddles<XS_RX>(tw, A.tw_x);
  __syncthreads();
  const int r = threadIdx.x / XS_RX, t = threadIdx.x % XS_RX;
  cx* sa = tw + XS_TWN(XS_RX) + (2 * r) * XS_XLINE;  // field a: stage and transpose scratch
  cx* sb = sa + XS_XLINE;                             // field2
  const size_t cta = blockIdx.x;
  const int e = (int)((cta * XS_XROWS) / XS_NY), y = (int)((cta * XS_XROWS + r) % XS_NY);
  const u32 blk = (u32)(A.block0 + e / A.ens1), el = (u32)(e % A.ens1);
  const size_t off = ((size_t)e * XS_F) * XS_NS + (size_t)y * XS_NX + t;
  XsWarpSync ws;
  // one field from HBM (K state) into its stage in x space
  auto load_x = [&](const cx* src, cx* st) {
    cx v[XS_F][XS_RX];
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) v[f][j] = src[off + (size_t)f * XS_NS + XS_RX * j];
#pragma unroll
    for (int f = 0; f < XS_F; ++f) xs_ifft4<XS_RX, 1, 1>(v[f], t, tw, st, ws);
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) st[(f * XS_RX + j) * XS_RX + t] = v[f][j];
  };
  // one stage back to HBM in the K state
  auto store_k = [&](cx* st, cx* dst) {
    cx v[XS_F][XS_RX];
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) v[f][j] = st[(f * XS_RX + j) * XS_RX + t];
    __syncwarp();  // the transforms reuse the stage as scratch
#pragma unroll
    for (int f = 0; f < XS_F; ++f) xs_fft4<XS_RX, 1, 1>(v[f], t, tw, st, ws);
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) dst[off + (size_t)f * XS_NS + XS_RX * j] = v[f][j];
  };
  load_x(A.field, sa);
  if (MODE != 4) load_x(A.field2, sb);
  __syncwarp();
  const real dt = (real)(A.dtr * 0.5);
  const real t0 = (real)A.t, t1 = (real)(A.t + A.dtr * 0.5), t2 = (real)(A.t + A.dtr);
  const real ws_ = (real)A.wscale;
  // noise of element j (site t + RX j of row y) for the draws (d0, d1 >= 0: coarse average)
  auto noise = [&](int j, int d0, int d1, real* w) {
#if XS_NW > 0
    const u32 s = (u32)(y * XS_NX + t + XS_RX * j);
    xs_normals_site<XS_NW>(w, s, el, (u32)d0, (u32)A.seq, A.seed, blk);
    if (d1 >= 0) {
      real w2[XS_NW];
      xs_normals_site<XS_NW>(w2, s, el, (u32)d1, (u32)A.seq, A.seed, blk);
#pragma unroll
      for (int c = 0; c < XS_NW; ++c) w[c] = (xs_mul_rn(w[c], ws_) + xs_mul_rn(w2[c], ws_)) * (real)0.5;
    } else {
#pragma unroll
      for (int c = 0; c < XS_NW; ++c) w[c] = w[c] * ws_;
    }
#else
    (void)j; (void)d0; (void)d1; w[0] = (real)0;
#endif
  };
#pragma unroll 1
  for (int j = 0; j < XS_RX; ++j) {
    real x, yy;
    xs_row_coords(y, t, j, x, yy);
    real w[XS_NW > 0 ? XS_NW : 1];
    noise(j, A.draw0, A.draw1, w);
    cx a[XS_F], b[XS_F], d[XS_F];
#pragma unroll
    for (int f = 0; f < XS_F; ++f) a[f] = sa[(f * XS_RX + j) * XS_RX + t];
    if (MODE == 4) {  // a1 = a + dt D(a, t)
      xs_deriv(a, w, (const cx*)nullptr, x, yy, (real)0, t0, A.params, (const cx*)nullptr, 0, 0, d);
#pragma unroll
      for (int f = 0; f < XS_F; ++f) sb[(f * XS_RX + j) * XS_RX + t] = a[f] + dt * d[f];
    } else if (MODE == 5) {
      cx a1[XS_F], a2[XS_F];
#pragma unroll
      for (int f = 0; f < XS_F; ++f) a1[f] = sb[(f * XS_RX + j) * XS_RX + t];
      xs_deriv(a1, w, (const cx*)nullptr, x, yy, (real)0, t1, A.params, (const cx*)nullptr, 0, 0, d);
#pragma unroll
      for (int f = 0; f < XS_F; ++f) a2[f] = a[f] + dt * d[f];
      xs_deriv(a2, w, (const cx*)nullptr, x, yy, (real)0, t1, A.params, (const cx*)nullptr, 0, 0, d);
#pragma unroll
      for (int f = 0; f < XS_F; ++f) {
        b[f] = a[f] + (real)2 * dt * d[f];  // a3
        sa[(f * XS_RX + j) * XS_RX + t] = (a1[f] + (real)2 * a2[f] + b[f] - a[f]) / (real)3;
        sb[(f * XS_RX + j) * XS_RX + t] = b[f];
      }
    } else {  // MODE 6: a = a + dt/3 D(a3, t + 2 dt), then the next step's pass 1
#pragma unroll
      for (int f = 0; f < XS_F; ++f) b[f] = sb[(f * XS_RX + j) * XS_RX + t];
      xs_deriv(b, w, (const cx*)nullptr, x, yy, (real)0, t2, A.params, (const cx*)nullptr, 0, 0, d);
#pragma unroll
      for (int f = 0; f < XS_F; ++f) {
        a[f] = a[f] + d[f] * dt / (real)3;
        sa[(f * XS_RX + j) * XS_RX + t] = a[f];
      }
      if (A.fuse) {
        noise(j, A.ndraw0, A.ndraw1, w);
        xs_deriv(a, w, (const cx*)nullptr, x, yy, (real)0, t2, A.params, (const cx*)nullptr, 0, 0, d);
#pragma unroll
        for (int f = 0; f < XS_F; ++f) sb[(f * XS_RX + j) * XS_RX + t] = a[f] + dt * d[f];
      }
    }
  }
  __syncwarp();
  if (MODE != 4) store_k(sa, A.field);
  if (MODE != 6 || A.fuse) store_k(sb, A.field2);
}

extern "C" __global__ void __launch_bounds__(256) xs_x_rk1(const XsStreamArgs A) { xs_rk4_row<4>(A); }
extern "C" __global__ void __launch_bounds__(256) xs_x_rk2(const XsStreamArgs A) { xs_rk4_row<5>(A); }
extern "C" __global__ void __launch_bounds__(256) xs_x_rk3(const XsStreamArgs A) { xs_rk4_row<6>(A); }

// ---- column pass ------------------------------------------------------------
// CTA = TX consecutive kx columns of one (trajectory, component); thread
// (c = tid % TX, t = tid / TX) holds y = t + RY*j of column c.
#define XS_SSMEM (XS_TWN(XS_RY) + XS_TX * XS_RY * XS_RY)

// FFT_y, x exp(L dt)^m, IFFT_y of one tile column held four-step style in v.
template <class Sync = XsBlockSync>
__device__ __forceinline__ void xs_col_tile(cx (&v)[XS_RY], int t, int c, int x0, int f, const cx* tw, cx* buf,
                                            const XsStreamArgs& A, Sync bs = Sync()) {
  xs_fft4<XS_RY, XS_TX, 0>(v, t, tw, buf, bs);
#if XS_SEP
  // separable L(kx, ky) = Lx(kx) + Ly(ky): exp(L dt) = ex[kx] * ey[ky] from two
  // 1D FP64 tables [NX] + [NY] (L1-resident) instead of the [NY][NX] table
  // The inverse transform's 1/NY (a power of two: exact, bit-identical to scaling its output)
  // rides on the FP64 propagator multiply.
  const double sc = 1.0 / (double)XS_NY;
  const double2* Pt = A.m == 2 ? A.prop2 : A.prop1;
  const double2 ex0 = __ldg(&Pt[x0 + c]);
  const double2 ex = make_double2(ex0.x * sc, ex0.y * sc);
  (void)f;
#else
  const double sc = 1.0 / (double)XS_NY;
  const double2* P = (A.m == 2 ? A.prop2 : A.prop1) + (XS_PROP_COMPS > 1 ? (size_t)f * XS_NS : 0);
#endif
#pragma unroll
  for (int k = 0; k < XS_RY; ++k) {
#if XS_SEP
    const double2 ey = __ldg(&Pt[XS_NX + t + XS_RY * k]);
    const double2 pr = make_double2(ey.x * ex.x - ey.y * ex.y, ey.x * ex.y + ey.y * ex.x);
    const double vr = (double)v[k].re, vi = (double)v[k].im;
#else
    const double2 pr = __ldg(&P[(size_t)(t + XS_RY * k) * XS_NX + x0 + c]);
    const double vr = (double)v[k].re * sc, vi = (double)v[k].im * sc;
#endif
    v[k] = mkcx((real)(vr * pr.x - vi * pr.y), (real)(vr * pr.y + vi * pr.x));
  }
  xs_ifft4u<XS_RY, XS_TX, 0>(v, t, tw, buf, bs);
}

// Column tile `tile` (over ntraj * F * NX/TX) by 256 threads tid = 0..255 with
// the shared memory `smem` (XS_SSMEM elements) and their barrier `bs`.
template <class Sync>
__device__ __forceinline__ void xs_col_core(const XsStreamArgs& A, int tid, size_t tile, cx* smem, Sync bs) {
  cx* tw = smem;
  xs_fill_twiddles<XS_RY, false>(tw, A.tw_y, tid, 256);  // xs_col_tile scales through the propagator
  const int c = tid % XS_TX, t = tid / XS_TX;
  cx* buf = tw + XS_TWN(XS_RY) + c;  // element (k, t) of column c at ((k*RY + t)*TX + c)
  constexpr int TILES = XS_NX / XS_TX;
  const int x0 = (int)(tile % TILES) * XS_TX;
  const size_t ef = tile / TILES;  // e * F + f
  cx* base = A.field + ef * XS_NS + x0 + c;
  cx v[XS_RY];
#pragma unroll
  for (int j = 0; j < XS_RY; ++j) v[j] = base[(size_t)(t + XS_RY * j) * XS_NX];
  bs();  // twiddles ready
  xs_col_tile(v, t, c, x0, (int)(ef % XS_F), tw, buf, A, bs);
#pragma unroll
  for (int j = 0; j < XS_RY; ++j) base[(size_t)(t + XS_RY * j) * XS_NX] = v[j];
}

// Minimum resident CTAs per SM (register budget) of the column pass.  FP32: 64 registers, four
// CTAs per SM.  FP64 lines hold 16 complex doubles per thread and spill at 64 or 80 registers, so
// FP64 builds take 128 (two CTAs per SM).  XSPDE_B200_DEFINES="-DXS_SPASS_MINB=n" overrides it.
#ifndef XS_SPASS_MINB
#define XS_SPASS_MINB (XS_FP64 ? 2 : 4)
#endif
extern "C" __global__ void __launch_bounds__(256, XS_SPASS_MINB) xs_s_pass(const XsStreamArgs A) {
  if ((size_t)blockIdx.x >= (size_t)A.ntraj * XS_F * (XS_NX / XS_TX)) {
    if (threadIdx.x == 0) atomicOr(A.status, 2);
    return;
  }
  if (!xs_smem_ok(XS_SSMEM * sizeof(cx), A.status)) return;
  xs_col_core(A, threadIdx.x, blockIdx.x, (cx*)xs_dsmem, XsBlockSync());
}

// ---- fused row + column pass ------------------------------------------------------
// Two independent halves of the trajectories one pass apart: one grid holds the
// row blocks of R (xs_x_nl) and the column tiles of C (xs_s_pass), interleaved
// by block index (row, column, row, ...), each CTA one role with the usual
// 256 threads.  As short column CTAs finish, the block scheduler refills their
// slots, so every SM keeps a mix of issue-bound row CTAs and HBM-bound column
// CTAs.
extern "C" __global__ void __launch_bounds__(256, XS_SPASS_MINB) xs_rc_pass(const XsStreamArgs R, const XsStreamArgs C) {
  const size_t nr = (size_t)R.ntraj * XS_NY / XS_XROWS, ncol = (size_t)C.ntraj * XS_F * (XS_NX / XS_TX);
  const size_t m = nr < ncol ? nr : ncol;
  const size_t i = blockIdx.x;
  const bool row = i < 2 * m ? (i & 1) == 0 : nr > ncol;
  const size_t idx = i < 2 * m ? i >> 1 : m + (i - 2 * m);
  if (row) {
    if (idx >= nr) {
      if (threadIdx.x == 0) atomicOr(R.status, 2);
      return;
    }
    if (!xs_smem_ok(XS_XSMEM * sizeof(cx), R.status)) return;
    xs_xpass_core<1>(R, threadIdx.x, idx, (cx*)xs_dsmem, XsBlockSync());
  } else {
    if (idx >= ncol) {
      if (threadIdx.x == 0) atomicOr(C.status, 2);
      return;
    }
    if (!xs_smem_ok(XS_SSMEM * sizeof(cx), C.status)) return;
    xs_col_core(C, threadIdx.x, idx, (cx*)xs_dsmem, XsBlockSync());
  }
}

// ---- column pass fed by the Tensor Memory Accelerator ---------------------------
// Persistent CTAs walk the tiles (TX columns x NY rows of one trajectory and
// component) with stride gridDim.x.  Thread 0 issues one 2D bulk tensor copy
// per tile (cp.async.bulk.tensor, box 2*TX reals x NY rows of the field viewed
// as [rows][2*NX] reals) into one of two shared-memory stages, completing on
// that stage's mbarrier; the tile after next is requested as soon as a stage
// has been read into registers, so HBM reads overlap the FFTs.  Results are
// stored straight from registers (128-byte row segments).  Arithmetic is that
// of xs_s_pass.  Every wait is bounded: on a timeout the CTA sets status bit 3,
// waits (bounded) for its copies in flight and returns.
struct __align__(64) XsTmap {
  unsigned long long w[16];
};

__device__ __forceinline__ u32 xs_smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool xs_mbar_wait(u32 bar, u32 parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    u32 ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void xs_tma_load_2d(const XsTmap* tm, u32 dst, u32 bar, int x, int y, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"((unsigned long long)tm), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

#define XS_STAGE_ELEMS (XS_NY * XS_TX)
#define XS_TSMEM_BYTES (2 * XS_STAGE_ELEMS * sizeof(cx) + XS_TWN(XS_RY) * sizeof(cx) + 16 + 128)

extern "C" __global__ void __launch_bounds__(256) xs_s_pass_tma(const XsStreamArgs A, const __grid_constant__ XsTmap tmap) {
  constexpr int TILES = XS_NX / XS_TX;
  const int ntiles = A.ntraj * XS_F * TILES;
  if (!xs_smem_ok(XS_TSMEM_BYTES, A.status)) return;
  unsigned char* base = (unsigned char*)(((size_t)xs_dsmem + 127) & ~(size_t)127);
  cx* stage = (cx*)base;                 // [2][NY][TX] (row-major tiles as the copies deliver them)
  cx* tw = stage + 2 * XS_STAGE_ELEMS;   // [RY*RY] twiddles
  const int c = threadIdx.x % XS_TX, t = threadIdx.x / XS_TX;
  unsigned long long* bars = (unsigned long long*)(tw + XS_TWN(XS_RY));
  const u32 bar0 = xs_smem_u32(&bars[0]);  // stage s completes on bar0 + 8 s
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  xs_fill_twiddles<XS_RY, false>(tw, A.tw_y);
  __syncthreads();
  const u32 bytes = (u32)(XS_STAGE_ELEMS * sizeof(cx));
  auto issue = [&](int tile, int sidx) {
    const int x0 = (tile % TILES) * XS_TX, ef = tile / TILES;
    xs_tma_load_2d(&tmap, xs_smem_u32(stage + sidx * XS_STAGE_ELEMS), bar0 + 8u * sidx, 2 * x0, ef * XS_NY, bytes);
  };
  if (threadIdx.x == 0) {
    if ((int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < ntiles) issue(blockIdx.x + gridDim.x, 1);
  }
  int i = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
    const int sidx = i & 1;
    const bool ok = xs_mbar_wait(bar0 + 8u * sidx, (u32)((i >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(A.status, 8);
        xs_mbar_wait(bar0 + 8u * sidx, (u32)((i >> 1) & 1));
        if (tile + (int)gridDim.x < ntiles) xs_mbar_wait(bar0 + 8u * (sidx ^ 1), (u32)(((i + 1) >> 1) & 1));
      }
      return;
    }
    cx v[XS_RY];
    cx* st = stage + sidx * XS_STAGE_ELEMS;
#pragma unroll
    for (int j = 0; j < XS_RY; ++j) v[j] = st[(t + XS_RY * j) * XS_TX + c];
    __syncthreads();  // stage sidx fully read: it becomes this tile's transpose scratch
    const int x0 = (tile % TILES) * XS_TX, ef = tile / TILES;
    xs_col_tile(v, t, c, x0, ef % XS_F, tw, st + c, A);
    cx* gb = A.field + (size_t)ef * XS_NS + x0 + c;
#pragma unroll
    for (int j = 0; j < XS_RY; ++j) gb[(size_t)(t + XS_RY * j) * XS_NX] = v[j];
    // the FFTs end with a barrier, so the scratch is free: refill it with the tile after next
    if (threadIdx.x == 0 && tile + 2 * (int)gridDim.x < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(tile + 2 * gridDim.x, sidx);
    }
  }
}

// ---- observation pass ---------------------------------------------------------
// CTA = (row group, block): OROWS rows of every trajectory of the block.
// Site observables: block sums in FP64 registers, written as block means.
// Reductions (Int/Ave): per-trajectory sums over the row group -> redpart.
#define XS_OSMEM (XS_TWN(XS_RX) + XS_OROWS * XS_RX * (XS_RX + 1))

extern "C" __global__ void __launch_bounds__(XS_OROWS * XS_RX) xs_x_obs(const XsStreamArgs A) {
  if ((int)blockIdx.x >= XS_NRG || (size_t)(blockIdx.y + 1) * A.ens1 > (size_t)A.ntraj) {
    if (threadIdx.x == 0) atomicOr(A.status, 2);
    return;
  }
  cx* smem = (cx*)xs_dsmem;
  __shared__ double wred[(XS_OROWS * XS_RX + 31) / 32][2 * (XS_NRED > 0 ? XS_NRED : 1)];
  cx* tw = smem;
  xs_fill_twiddles<XS_RX>(tw, A.tw_x);
  __syncthreads();
  const int r = threadIdx.x / XS_RX, t = threadIdx.x % XS_RX;
  cx* buf = tw + XS_TWN(XS_RX) + r * XS_RX * (XS_RX + 1);
  const int rg = blockIdx.x;       // row group
  const int b = blockIdx.y;        // block within the launch
  const int y = rg * XS_OROWS + r;
  const real tt = (real)A.t;
  XsWarpSync ws;
#if XS_NOUT_SITE > 0
  // compensated sums over the block's trajectories (xs_kadd)
  double sr[XS_NOUT_SITE][XS_RX], si[XS_NOUT_SITE][XS_RX], cr[XS_NOUT_SITE][XS_RX], ci[XS_NOUT_SITE][XS_RX];
#pragma unroll
  for (int k = 0; k < XS_NOUT_SITE; ++k)
#pragma unroll
    for (int j = 0; j < XS_RX; ++j) sr[k][j] = si[k][j] = cr[k][j] = ci[k][j] = 0;
#endif
  // the block's trajectories el = z, z + Z, ... (Z = gridDim.z splits of each block, for
  // latency hiding; xs_x_obs_combine adds the splits)
  for (int el = blockIdx.z; el < A.ens1; el += gridDim.z) {
    const int e = b * A.ens1 + el;
    cx v[XS_F][XS_RX];
    const cx* base = A.field + ((size_t)e * XS_F) * XS_NS + (size_t)y * XS_NX + t;
#pragma unroll
    for (int f = 0; f < XS_F; ++f)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j) v[f][j] = base[(size_t)f * XS_NS + XS_RX * j];
#pragma unroll
    for (int f = 0; f < XS_F; ++f) xs_ifft4<XS_RX, 1, 1>(v[f], t, tw, buf, ws);
    {  // a diverged trajectory is reported (status bit 0) at every observation, not only by xs_x_final
      bool bad = false;
#pragma unroll
      for (int f = 0; f < XS_F; ++f)
#pragma unroll
        for (int j = 0; j < XS_RX; ++j) bad |= !isfinite((double)v[f][j].re) || !isfinite((double)v[f][j].im);
      if (bad) atomicOr(A.status, 1);
    }
#if XS_NRED > 0
    double acc[2 * XS_NRED];
#pragma unroll
    for (int k = 0; k < 2 * XS_NRED; ++k) acc[k] = 0;
#endif
#pragma unroll
    for (int j = 0; j < XS_RX; ++j) {
      real x, yy;
      xs_row_coords(y, t, j, x, yy);
      cx a[XS_F];
#pragma unroll
      for (int f = 0; f < XS_F; ++f) a[f] = v[f][j];
#if XS_NRED > 0
      cx rr[XS_NRED];
      xs_integrands(a, a, (const cx*)nullptr, (const cx*)nullptr, 0, 0, t + XS_RX * j, y, 0, x, yy, (real)0, tt, A.params, rr);
#pragma unroll
      for (int k = 0; k < XS_NRED; ++k) { acc[2 * k] += (double)rr[k].re; acc[2 * k + 1] += (double)rr[k].im; }
#endif
#if XS_NOUT_SITE > 0
      cx o[XS_NOUT_SITE];
      xs_obs_site(a, a, (const cx*)nullptr, (const cx*)nullptr, 0, 0, (const cx*)nullptr, x, yy, (real)0, t + XS_RX * j, y, 0, tt, A.params, o);
#pragma unroll
      for (int k = 0; k < XS_NOUT_SITE; ++k) {
        xs_kadd(sr[k][j], cr[k][j], (double)o[k].re);
        if (xs_ocplx_site(k)) xs_kadd(si[k][j], ci[k][j], (double)o[k].im);
      }
#endif
    }
#if XS_NRED > 0
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 2 * XS_NRED; ++k) {
      const double s = xs_warp_sum(acc[k]);
      if (lane == 0) wred[warp][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < XS_NRED) {
      double re = 0, im = 0;
      for (int q = 0; q < (XS_OROWS * XS_RX + 31) / 32; ++q) {
        re += wred[q][2 * threadIdx.x];
        im += wred[q][2 * threadIdx.x + 1];
      }
      A.redpart[((size_t)e * XS_NRG + rg) * XS_NRED + threadIdx.x] = make_double2(re, im);
    }
    __syncthreads();
#endif
  }
#if XS_NOUT_SITE > 0
  if (gridDim.z == 1) {
    const double inv = 1.0 / (double)A.ens1;
    double2* out = A.av + ((size_t)b * A.npoints + A.n) * XS_OBS_STRIDE;
#pragma unroll
    for (int k = 0; k < XS_NOUT_SITE; ++k)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j)
        out[(size_t)k * XS_NS + (size_t)y * XS_NX + t + XS_RX * j] =
            make_double2((sr[k][j] + cr[k][j]) * inv, (si[k][j] + ci[k][j]) * inv);
  } else {
    double2* out = A.opart + ((size_t)blockIdx.z * gridDim.y + b) * ((size_t)XS_NOUT_SITE * XS_NS);
#pragma unroll
    for (int k = 0; k < XS_NOUT_SITE; ++k)
#pragma unroll
      for (int j = 0; j < XS_RX; ++j)
        out[(size_t)k * XS_NS + (size_t)y * XS_NX + t + XS_RX * j] =
            make_double2(sr[k][j] + cr[k][j], si[k][j] + ci[k][j]);
  }
#endif
}

// Scalar observables from the per-trajectory reductions of the row groups.
extern "C" __global__ void __launch_bounds__(256) xs_stream_scalar(const XsStreamArgs A) { xs_scalar_body<XS_NRG>(A); }
