// Streaming-path kernels for 3D lattices with non-periodic boundaries in every
// space dimension (Simulator/xpath.m:29-86 with Applications/SDE/MP.m and the
// DST/DCT branch of Applications/SPDE/xprop.m:18-42, whose transforms are
// Applications/SPDE/xdct1.m, xdst1.m, xdct2.m, xdct3.m, xdst2.m, xdst3.m).
//
// Field layout in HBM: F[e][z][y][x], x fastest, complex `real`, one field
// component.  Between passes the field is held transformed along x and y
// ("K state": kx, ky, z).  One MP step (merged with its neighbour's half step):
//   xs_z_pass   z-line pass: T_z, multiply by exp(L dtr/2)^m (FP64 table, m = 2
//               merges the previous step's second half with this step's first
//               half), T_z^-1
//   xs_p_nl     plane pass: T_y^-1, T_x^-1, midpoint iterations with the drift,
//               Philox noise and the Dirichlet mask, 2a - a0, T_x, T_y
// Each pass reads and writes the field once: 4 N F s bytes per trajectory-step.
//
// Every transform is the reference's real matrix (built on the host in FP64 by
// applying the reference's transform to unit vectors), applied densely from
// shared memory: out[k] = sum_n M[n][k] in[n].  Each matrix of these transforms
// is mirror-symmetric about a centre C in N-1, N-2 or N (DCT-I and DST-I: N - 1;
// DCT-II/III: N - 2 with row or column N - 1 zero; DST-II/III: N with row or
// column 0 zero), which halves its multiply-adds:
//   input fold, M[C-n][k] = (-1)^(k+p) M[n][k]: u_n = in[n] + in[C-n] and
//     v_n = in[n] - in[C-n] over the first half of the rows; outputs with k + p
//     even sum M[n][k] u_n, the others M[n][k] v_n (DCT-I, DST-I, DCT-II, DST-II);
//   output fold, M[n][C-k] = (-1)^(n+p) M[n][k]: E_k sums the inputs with n + p
//     even, O_k the others, over the first half of the outputs; out[k] = E + O,
//     out[C-k] = E - O (DCT-III, DST-III).
// The host packs the half of each matrix that is read (rows for an input fold,
// columns for an output fold) and sets its entries that the symmetry makes zero
// to exactly zero.
//
// Passes are persistent: gridDim.x CTAs walk the planes (or z-line tiles) with
// stride gridDim.x, so each CTA stages its matrices in shared memory once.
#pragma once

#define XS3_N1 XS_N1
#define XS3_N2 XS_N2
#define XS3_N3 XS_N3
#define XS3_NP (XS_N1 * XS_N2)         // sites per plane
// XS3_LSX, XS3_LSQ (host): row strides of the plane and of the z-line tile in shared memory, in
// complex elements; even in FP32, so that four consecutive elements of a row are one pair of
// 16-byte loads
#define XS_NRG XS_N3                   // reduction parts per trajectory: one per plane

// Matrix i (0 x fwd, 1 x inv, 2 y fwd, 3 y inv, 4 z fwd, 5 z inv) in A.mat at offset
// XS3_MOFFi; XS3_FOLDi = 0 (full N x N), 1 (input fold: N/2 packed rows of N) or 2 (output
// fold: N rows of N/2 packed columns), about centre XS3_CENi with parity XS3_PARi.
template <int I> struct Xs3Mat;
#define XS3_MAT(I, NN)                                                                                  \
  template <> struct Xs3Mat<I> {                                                                       \
    static constexpr int N = NN, OFF = XS3_MOFF##I, FOLD = XS3_FOLD##I, C = XS3_CEN##I, PAR = XS3_PAR##I; \
  };
XS3_MAT(0, XS_N1)
XS3_MAT(1, XS_N1)
XS3_MAT(2, XS_N2)
XS3_MAT(3, XS_N2)
XS3_MAT(4, XS_N3)
XS3_MAT(5, XS_N3)
// reals of shared memory a matrix occupies (the packed half when folded)
template <int I> __host__ __device__ constexpr int xs3_msize() {
  return Xs3Mat<I>::FOLD ? Xs3Mat<I>::N * (Xs3Mat<I>::N / 2) : Xs3Mat<I>::N * Xs3Mat<I>::N;
}

// Copy matrix I into shared memory (all threads of the CTA; caller syncs).
template <int I>
__device__ __forceinline__ void xs3_stage_matrix(real* dst, const real* __restrict__ mat) {
  const real* src = mat + Xs3Mat<I>::OFF;
  for (int i = threadIdx.x; i < xs3_msize<I>(); i += blockDim.x) dst[i] = src[i];
}

// Four consecutive reals of a shared-memory matrix row (16- or 32-byte aligned).
__device__ __forceinline__ void xs3_load4(const real* p, real (&m)[4]) {
  if constexpr (sizeof(real) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    m[0] = q.x;
    m[1] = q.y;
    m[2] = q.z;
    m[3] = q.w;
  } else {
    const double2 q0 = *reinterpret_cast<const double2*>(p);
    const double2 q1 = *reinterpret_cast<const double2*>(p + 2);
    m[0] = q0.x;
    m[1] = q0.y;
    m[2] = q1.x;
    m[3] = q1.y;
  }
}

// Two consecutive complex elements (16-byte aligned in FP32).
__device__ __forceinline__ void xs3_load2(const cx* p, cx& a, cx& b) {
  if constexpr (sizeof(real) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    a = mkcx((real)q.x, (real)q.y);
    b = mkcx((real)q.z, (real)q.w);
  } else {
    a = p[0];
    b = p[1];
  }
}

// Row of the folded index j: the u row (input fold) or the output (output fold), and its
// partner C - r, or the zero row/column slot when j is its own partner.
template <int N, int C> __device__ __forceinline__ constexpr int xs3_fr(int j) { return j + (C == N ? 1 : 0); }
template <int N, int C> __device__ __forceinline__ constexpr int xs3_fp(int j) {
  return C - xs3_fr<N, C>(j) != xs3_fr<N, C>(j) ? C - xs3_fr<N, C>(j) : (C == N ? 0 : N - 1);
}

// In-place dense transform of the NL lines of length ND held in `buf` by the
// 256 threads of the CTA with the matrix I staged at Ms.  FORM_R: element n of
// line l at buf[n*LS + l] (lines are columns); otherwise at buf[l*LS + n]
// (lines are rows).  Each active thread computes 4 outputs of 4 lines in
// registers; a barrier separates all reads from the writes.
template <int I, int NL, int LS, bool FORM_R>
__device__ __forceinline__ void xs3_dense(cx* buf, const real* __restrict__ Ms, int tid) {
  constexpr int ND = Xs3Mat<I>::N, FOLD = Xs3Mat<I>::FOLD, C = Xs3Mat<I>::C, PAR = Xs3Mat<I>::PAR;
  constexpr int H = ND / 2;
  auto idx = [](int n, int l) { return FORM_R ? n * LS + l : l * LS + n; };
  // four consecutive lines of element n: two 16-byte loads when the lines are columns
  auto lines4 = [&](int n, int l0, cx (&x)[4]) {
    if constexpr (FORM_R) {
      xs3_load2(buf + n * LS + l0, x[0], x[1]);
      xs3_load2(buf + n * LS + l0 + 2, x[2], x[3]);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) x[j] = buf[(l0 + j) * LS + n];
    }
  };
  if constexpr (FOLD == 1) {
    for (int i = tid; i < H * NL; i += 256) {
      // consecutive threads take consecutive shared-memory words
      const int j = FORM_R ? i / NL : i % H, l = FORM_R ? i % NL : i / H;
      const int r = xs3_fr<ND, C>(j), q = xs3_fp<ND, C>(j);
      const bool self = C - r == r;  // its own partner: v is multiplied by zeros only
      const cx a = buf[idx(r, l)], b = self ? mkcx((real)0, (real)0) : buf[idx(q, l)];
      buf[idx(r, l)] = a + b;
      buf[idx(q, l)] = a - b;
    }
    __syncthreads();
  }
  constexpr int NOUT = FOLD == 2 ? H : ND;  // outputs computed per line (the first half when folded)
  constexpr int NKG = NOUT / 4, NT = NKG * (NL / 4);
  static_assert(NT <= 256, "one output tile per thread");
  const bool act = tid < NT;
  const int k0 = 4 * (tid % NKG), l0 = 4 * (tid / NKG);
  real ar[4][4], ai[4][4], br[4][4], bi[4][4];  // b: the odd-parity sums of an output fold
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int j = 0; j < 4; ++j) ar[q][j] = ai[q][j] = br[q][j] = bi[q][j] = 0;
  auto fma44 = [](real (&r)[4][4], real (&im)[4][4], const real (&m)[4], const cx (&x)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        r[q][j] += m[q] * x[j].re;
        im[q][j] += m[q] * x[j].im;
      }
  };
  if (act) {
    if constexpr (FOLD == 2) {
      // E (n + PAR even) into ar/ai, O into br/bi; n runs in pairs (even n first)
#pragma unroll 2
      for (int n = 0; n < ND; n += 2) {
        cx x0[4], x1[4];
        lines4(n, l0, x0);
        lines4(n + 1, l0, x1);
        real m0[4], m1[4];
        xs3_load4(Ms + n * H + k0, m0);
        xs3_load4(Ms + (n + 1) * H + k0, m1);
        if constexpr (PAR == 0) {
          fma44(ar, ai, m0, x0);
          fma44(br, bi, m1, x1);
        } else {
          fma44(br, bi, m0, x0);
          fma44(ar, ai, m1, x1);
        }
      }
    } else if constexpr (!FORM_R && (FOLD == 0 || C == ND - 1)) {
      // rows are lines: two consecutive elements (and their mirror pair) per 16-byte load
#pragma unroll 2
      for (int n = 0; n < (FOLD ? H : ND); n += 2) {
        cx x0[4], x1[4], d0[4], d1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          xs3_load2(buf + (l0 + j) * LS + n, x0[j], x1[j]);
          if constexpr (FOLD) xs3_load2(buf + (l0 + j) * LS + ND - 2 - n, d1[j], d0[j]);
        }
        real m0[4], m1[4];
        xs3_load4(Ms + n * ND + k0, m0);
        xs3_load4(Ms + (n + 1) * ND + k0, m1);
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const bool odd = FOLD && ((q + PAR) & 1);  // k0 is a multiple of 4
            const cx v0 = odd ? d0[j] : x0[j], v1 = odd ? d1[j] : x1[j];
            ar[q][j] += m0[q] * v0.re + m1[q] * v1.re;
            ai[q][j] += m0[q] * v0.im + m1[q] * v1.im;
          }
      }
    } else {
#pragma unroll 4
      for (int n = 0; n < (FOLD ? H : ND); ++n) {
        cx x[4], xd[4];
        if constexpr (FOLD) {
          lines4(xs3_fr<ND, C>(n), l0, x);
          lines4(xs3_fp<ND, C>(n), l0, xd);
        } else {
          lines4(n, l0, x);
        }
        real m[4];
        xs3_load4(Ms + n * ND + k0, m);
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const cx v = (FOLD && ((q + PAR) & 1)) ? xd[j] : x[j];  // k0 is a multiple of 4
            ar[q][j] += m[q] * v.re;
            ai[q][j] += m[q] * v.im;
          }
      }
    }
  }
  __syncthreads();
  if (act) {
    if constexpr (FOLD == 2) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = xs3_fr<ND, C>(k0 + q), kp = C - k;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          buf[idx(k, l0 + j)] = mkcx(ar[q][j] + br[q][j], ai[q][j] + bi[q][j]);
          if (kp != k) buf[idx(kp, l0 + j)] = mkcx(ar[q][j] - br[q][j], ai[q][j] - bi[q][j]);
        }
      }
      if (C != ND - 1 && k0 == 0)  // the zero output (row or column N-1, or 0)
#pragma unroll
        for (int j = 0; j < 4; ++j) buf[idx(C == ND ? 0 : ND - 1, l0 + j)] = mkcx((real)0, (real)0);
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int j = 0; j < 4; ++j) buf[idx(k0 + q, l0 + j)] = mkcx(ar[q][j], ai[q][j]);
    }
  }
  __syncthreads();
}

// ---- asynchronous staging ----------------------------------------------------------
// The persistent passes copy the next plane (or z-line tile) into a second shared-memory
// buffer with cp.async while the current one is transformed; copies of 16 bytes (two FP32 or
// one FP64 complex element), one commit group per fetch, waited for at the top of the next
// iteration.
__device__ __forceinline__ void xs3_cp16(cx* dst, const cx* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((u32)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void xs3_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void xs3_cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// ROWS rows of W complex elements, source row stride GS, into shared rows of stride LS.
template <int ROWS, int W, size_t GS, int LS>
__device__ __forceinline__ void xs3_fetch(cx* dst, const cx* __restrict__ src, int tid) {
  constexpr int E = 16 / (int)sizeof(cx);  // elements per copy
  static_assert(W % E == 0, "rows of whole 16-byte copies");
  for (int i = tid; i < ROWS * (W / E); i += 256) {
    const int r = i / (W / E), c = (i % (W / E)) * E;
    xs3_cp16(dst + r * LS + c, src + (size_t)r * GS + c);
  }
  xs3_cp_commit();
}

// ---- plane passes ---------------------------------------------------------------
// Shared memory: the matrices of the pass (xs3_psmem<MODE>() reals), then two
// planes P[y][x] (row stride XS3_LSX): the current one and the next, in flight.
__device__ __forceinline__ void xs3_coords(int i1, int i2, int i3, real& x, real& y, real& z) {
  x = (real)(XS_O1 + XS_DX1 * (double)i1);
  y = (real)(XS_O2 + XS_DX2 * (double)i2);
  z = (real)(XS_O3 + XS_DX3 * (double)i3);
}

// MODE 0: initial field (expression or a_in), stored in x space: its Dirichlet
//         boundary values, which no transform keeps, are observed at the first
//         output time as the reference observes them
// MODE 2: x space -> K state (T_x, T_y)
// MODE 1: one MP step (K state in, K state out)
// MODE 3: K state (or x space, A.xspace) -> x-space a_out (FP64)
// matrices staged: inverse x and y (MODE 1, 3), forward x and y (MODE 1, 2)
template <int MODE> __host__ __device__ constexpr int xs3_pinv() {
  return (MODE == 1 || MODE == 3) ? xs3_msize<1>() + xs3_msize<3>() : 0;
}
template <int MODE> __host__ __device__ constexpr int xs3_psmem() {
  return xs3_pinv<MODE>() + ((MODE == 1 || MODE == 2) ? xs3_msize<0>() + xs3_msize<2>() : 0);
}

// One MP step of the sites of plane z held in P (x space, row stride LS; NT threads): noise, midpoint
// iterations at t + dtr/2 with the Dirichlet mask (Applications/SDE/MP.m:13-23,
// Simulator/xsetbound.m), 2a - a0, written back in place.
template <int LS = XS3_LSX, int NT = 256>
__device__ __forceinline__ void xs3_mp_sites(const XsStreamArgs& A, cx* P, int e, int z, int tid) {
  const u32 blk = (u32)(A.block0 + e / A.ens1), el = (u32)(e % A.ens1);
  const real h = (real)(A.dtr * 0.5);
  const real tm = (real)(A.t + A.dtr * 0.5);
  const real ws = (real)A.wscale;
  auto site = [&](int i1, int i2, const real* w) {
    real x, y, zz;
    xs3_coords(i1, i2, z, x, y, zz);
    cx a0[1], a[1], d[1];
    a0[0] = a[0] = P[i2 * LS + i1];
#if XS_DSPLIT
    // a = (a0 + h inv) + h dep(a): the drift's field-independent terms once per site
    cx c0;
    xs_deriv_c0(a, a0, h, w, (const cx*)nullptr, x, y, zz, tm, A.params, (const cx*)nullptr, 0, 0, &c0);
#endif
#pragma unroll
    for (int it = 0; it < XS_ITER; ++it) {
#if XS_DSPLIT
      xs_deriv_step(a, &c0, h, w, (const cx*)nullptr, x, y, zz, tm, A.params, (const cx*)nullptr, 0, 0, d);
      a[0] = d[0];
#else
      xs_deriv(a, w, (const cx*)nullptr, x, y, zz, tm, A.params, (const cx*)nullptr, 0, 0, d);
      a[0] = a0[0] + h * d[0];
#endif
#if XS_SETBOUND
      if (xs_dirichlet(0, i1, i2, z)) a[0] = mkcx((real)0, (real)0);
#endif
    }
    P[i2 * LS + i1] = (real)2 * a[0] - a0[0];
  };
#if XS_NW > 0 && XS_PAIRED(XS_NW)
  // one Philox call per pair of sites (x, x + N1/2) of a row
  constexpr int H = XS3_N1 / 2;
#pragma unroll 1
  for (int pi = tid; pi < XS3_NP / 2; pi += NT) {
    const int i2 = pi / H, xl = pi % H;
    const u32 pidx = (u32)xl + (u32)H * (u32)(i2 + XS3_N2 * z);
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
    site(xl, i2, wl);
    site(xl + H, i2, wh);
  }
#else
#pragma unroll 1
  for (int i = tid; i < XS3_NP; i += NT) {
    const int i2 = i / XS3_N1, i1 = i % XS3_N1;
    real w[XS_NW > 0 ? XS_NW : 1];
#if XS_NW > 0
    const u32 s = (u32)(i + XS3_NP * z);
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
#else
    w[0] = (real)0;
#endif
    site(i1, i2, w);
  }
#endif
}

// Initial field in x space, one thread per site (no shared memory).
__device__ __forceinline__ void xs3_initial_pass(const XsStreamArgs& A) {
  const size_t nsites = (size_t)A.ntraj * XS_NS;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nsites; i += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(i / XS_NS);
    const size_t s = i % XS_NS;
    cx a[1];
    if (A.a_in) {
      const double2 q = A.a_in[i];
      a[0] = mkcx((real)q.x, (real)q.y);
    } else {
      const int i1 = (int)(s % XS3_N1), i2 = (int)((s / XS3_N1) % XS3_N2), i3 = (int)(s / XS3_NP);
      const u32 blk = (u32)(A.block0 + e / A.ens1), el = (u32)(e % A.ens1);
      real x, y, zz;
      xs3_coords(i1, i2, i3, x, y, zz);
      real vv[XS_NV > 0 ? XS_NV : 1];
#if XS_NV > 0
      xs_normals_site<XS_NV>(vv, (u32)s, el, 0u, (u32)A.seq, A.seed, blk);
#pragma unroll
      for (int c = 0; c < XS_NV; ++c) vv[c] *= (real)A.vscale;
#else
      vv[0] = (real)0;
#endif
      xs_initial(vv, (const cx*)nullptr, x, y, zz, A.params, a);
    }
    A.field[i] = a[0];
  }
}

template <int MODE>
__device__ __forceinline__ void xs3_plane_pass(const XsStreamArgs& A) {
  constexpr size_t need = (size_t)xs3_psmem<MODE>() * sizeof(real) + 2 * (size_t)XS3_N2 * XS3_LSX * sizeof(cx);
  if (!xs_smem_ok(need, A.status)) return;
  real* sm = (real*)xs_dsmem;
  real* Mxi = sm;
  real* Myi = Mxi + (xs3_pinv<MODE>() ? xs3_msize<1>() : 0);
  real* Mxf = sm + xs3_pinv<MODE>();
  real* Myf = Mxf + ((MODE == 1 || MODE == 2) ? xs3_msize<0>() : 0);
  cx* P = (cx*)(sm + xs3_psmem<MODE>());  // the plane being transformed
  cx* Q = P + XS3_N2 * XS3_LSX;            // the next plane, in flight
  const int tid = threadIdx.x;
  const size_t nplanes = (size_t)A.ntraj * XS3_N3;
  if (blockIdx.x < nplanes) xs3_fetch<XS3_N2, XS3_N1, XS3_N1, XS3_LSX>(P, A.field + blockIdx.x * XS3_NP, tid);
  if constexpr (MODE == 1 || MODE == 3) {
    xs3_stage_matrix<1>(Mxi, A.mat);
    xs3_stage_matrix<3>(Myi, A.mat);
  }
  if constexpr (MODE == 1 || MODE == 2) {
    xs3_stage_matrix<0>(Mxf, A.mat);
    xs3_stage_matrix<2>(Myf, A.mat);
  }
  bool bad = false;
  for (size_t pl = blockIdx.x; pl < nplanes; pl += gridDim.x) {
    const int e = (int)(pl / XS3_N3), z = (int)(pl % XS3_N3);
    cx* g = A.field + pl * XS3_NP;  // F = 1: plane pl of the [e][z] planes
    xs3_cp_wait_all();
    __syncthreads();  // this plane (and, the first time, the matrices) staged; Q free
    if (pl + gridDim.x < nplanes)
      xs3_fetch<XS3_N2, XS3_N1, XS3_N1, XS3_LSX>(Q, A.field + (pl + gridDim.x) * XS3_NP, tid);
    if (MODE == 1 || (MODE == 3 && !A.xspace)) {
      xs3_dense<3, XS3_N1, XS3_LSX, true>(P, Myi, tid);   // T_y^-1: lines are the x columns
      xs3_dense<1, XS3_N2, XS3_LSX, false>(P, Mxi, tid);  // T_x^-1: lines are the y rows
    }
    if constexpr (MODE == 1) {
      xs3_mp_sites(A, P, e, z, tid);
      __syncthreads();
    }
    if constexpr (MODE == 3) {
      for (int i = tid; i < XS3_NP; i += 256) {
        const cx q = P[(i / XS3_N1) * XS3_LSX + i % XS3_N1];
        bad |= !isfinite((double)q.re) || !isfinite((double)q.im);
        if (A.a_out) A.a_out[(size_t)e * XS_NS + (size_t)i + (size_t)XS3_NP * z] = make_double2((double)q.re, (double)q.im);
      }
    } else {
      xs3_dense<0, XS3_N2, XS3_LSX, false>(P, Mxf, tid);  // T_x
      xs3_dense<2, XS3_N1, XS3_LSX, true>(P, Myf, tid);   // T_y
      for (int i = tid; i < XS3_NP; i += 256) g[i] = P[(i / XS3_N1) * XS3_LSX + i % XS3_N1];
    }
    cx* const t = P;  // the next iteration's barrier orders these reads before Q's refill
    P = Q;
    Q = t;
  }
  if (bad) atomicOr(A.status, 1);
}

extern "C" __global__ void __launch_bounds__(256) xs_p_init(const XsStreamArgs A) { xs3_initial_pass(A); }
extern "C" __global__ void __launch_bounds__(256) xs_p_tok(const XsStreamArgs A) { xs3_plane_pass<2>(A); }
extern "C" __global__ void __launch_bounds__(256) xs_p_nl(const XsStreamArgs A) { xs3_plane_pass<1>(A); }
extern "C" __global__ void __launch_bounds__(256) xs_p_final(const XsStreamArgs A) { xs3_plane_pass<3>(A); }

// ---- z-line pass ----------------------------------------------------------------
// Tile = XS3_QT consecutive (kx, ky) columns of one trajectory by N3 z points:
// T[z][q] (row stride XS3_LSQ), each row one 8*QT-byte (FP32) run of a plane.
// T_z, multiply by exp(L dtr/2)^m at (kx, ky, kz) (site order of the FP64
// table), T_z^-1.  Shared memory: the two z matrices, then two tiles (the current
// one and the next, in flight).
__host__ __device__ constexpr int xs3_zsmem() { return xs3_msize<4>() + xs3_msize<5>(); }

extern "C" __global__ void __launch_bounds__(256) xs_z_pass(const XsStreamArgs A) {
  constexpr size_t need = (size_t)xs3_zsmem() * sizeof(real) + 2 * (size_t)XS3_N3 * XS3_LSQ * sizeof(cx);
  if (!xs_smem_ok(need, A.status)) return;
  real* Mzf = (real*)xs_dsmem;
  real* Mzi = Mzf + xs3_msize<4>();
  cx* T = (cx*)(Mzf + xs3_zsmem());  // the tile being transformed
  cx* U = T + XS3_N3 * XS3_LSQ;      // the next tile, in flight
  const int tid = threadIdx.x;
  constexpr int TPT = XS3_NP / XS3_QT;  // tiles per trajectory
  const size_t ntiles = (size_t)A.ntraj * TPT;
  auto origin = [&](size_t tile) { return A.field + (tile / TPT) * XS_NS + (tile % TPT) * XS3_QT; };
  if (blockIdx.x < ntiles) xs3_fetch<XS3_N3, XS3_QT, XS3_NP, XS3_LSQ>(T, origin(blockIdx.x), tid);
  xs3_stage_matrix<4>(Mzf, A.mat);
  xs3_stage_matrix<5>(Mzi, A.mat);
  const double2* __restrict__ tab = A.m == 2 ? A.prop2 : A.prop1;
  for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int q0 = (int)(tile % TPT) * XS3_QT;
    cx* g = origin(tile);
    xs3_cp_wait_all();
    __syncthreads();  // this tile (and, the first time, the matrices) staged; U free
    if (tile + gridDim.x < ntiles) xs3_fetch<XS3_N3, XS3_QT, XS3_NP, XS3_LSQ>(U, origin(tile + gridDim.x), tid);
    xs3_dense<4, XS3_QT, XS3_LSQ, true>(T, Mzf, tid);  // T_z
#if XS_HAS_PROP
    for (int i = tid; i < XS3_N3 * XS3_QT; i += 256) {
      const int kz = i / XS3_QT, q = i % XS3_QT;
      const double2 pr = tab[(size_t)q0 + q + (size_t)XS3_NP * kz];
      const cx v = T[kz * XS3_LSQ + q];
      const double vr = (double)v.re, vi = (double)v.im;
      T[kz * XS3_LSQ + q] = mkcx((real)(vr * pr.x - vi * pr.y), (real)(vr * pr.y + vi * pr.x));
    }
    __syncthreads();
#endif
    xs3_dense<5, XS3_QT, XS3_LSQ, true>(T, Mzi, tid);  // T_z^-1
    for (int i = tid; i < XS3_N3 * XS3_QT; i += 256) {
      const int z = i / XS3_QT, q = i % XS3_QT;
      g[(size_t)z * XS3_NP + q] = T[z * XS3_LSQ + q];
    }
    cx* const t = T;  // the next iteration's barrier orders these reads before U's refill
    T = U;
    U = t;
  }
}

// ---- observation pass -------------------------------------------------------------
// CTA = (plane z, block b, split): the trajectories el = split, split + Z, ... of
// block b (Z = gridDim.z; xs_x_obs_combine adds the splits).  Each plane is
// taken back to x space (T_y^-1, T_x^-1); site observables are summed in FP64
// registers (thread tid holds sites tid + 256 j), integrands of Int/Ave are
// summed per trajectory over the plane into redpart[e][z].
#define XS3_J ((XS3_NP + 255) / 256)

extern "C" __global__ void __launch_bounds__(256) xs_p_obs(const XsStreamArgs A) {
  constexpr size_t need = (size_t)xs3_pinv<3>() * sizeof(real) + (size_t)XS3_N2 * XS3_LSX * sizeof(cx);
  if ((int)blockIdx.x >= XS3_N3 || (size_t)(blockIdx.y + 1) * A.ens1 > (size_t)A.ntraj) {
    if (threadIdx.x == 0) atomicOr(A.status, 2);
    return;
  }
  if (!xs_smem_ok(need, A.status)) return;
  __shared__ double wred[8][2 * (XS_NRED > 0 ? XS_NRED : 1)];
  real* Mxi = (real*)xs_dsmem;
  real* Myi = Mxi + xs3_msize<1>();
  cx* P = (cx*)(Mxi + xs3_pinv<3>());
  xs3_stage_matrix<1>(Mxi, A.mat);
  xs3_stage_matrix<3>(Myi, A.mat);
  const int tid = threadIdx.x, z = blockIdx.x, b = blockIdx.y;
  const real tt = (real)A.t;
#if XS_NOUT_SITE > 0
  double sr[XS_NOUT_SITE][XS3_J], si[XS_NOUT_SITE][XS3_J];
#pragma unroll
  for (int k = 0; k < XS_NOUT_SITE; ++k)
#pragma unroll
    for (int j = 0; j < XS3_J; ++j) sr[k][j] = si[k][j] = 0;
#endif
  bool bad = false;
  for (int el = blockIdx.z; el < A.ens1; el += gridDim.z) {
    const int e = b * A.ens1 + el;
    const cx* g = A.field + ((size_t)e * XS3_N3 + z) * XS3_NP;
    for (int i = tid; i < XS3_NP; i += 256) P[(i / XS3_N1) * XS3_LSX + i % XS3_N1] = g[i];
    __syncthreads();
    if (!A.xspace) {
      xs3_dense<3, XS3_N1, XS3_LSX, true>(P, Myi, tid);
      xs3_dense<1, XS3_N2, XS3_LSX, false>(P, Mxi, tid);
    }
#if XS_NRED > 0
    double acc[2 * XS_NRED];
#pragma unroll
    for (int k = 0; k < 2 * XS_NRED; ++k) acc[k] = 0;
#endif
#pragma unroll
    for (int j = 0; j < XS3_J; ++j) {
      const int i = tid + 256 * j;
      if (XS3_NP % 256 == 0 || i < XS3_NP) {
        const int i2 = i / XS3_N1, i1 = i % XS3_N1;
        cx a[1];
        a[0] = P[i2 * XS3_LSX + i1];
        bad |= !isfinite((double)a[0].re) || !isfinite((double)a[0].im);
        real x, y, zz;
        xs3_coords(i1, i2, z, x, y, zz);
#if XS_NRED > 0
        cx rr[XS_NRED];
        xs_integrands(a, a, (const cx*)nullptr, (const cx*)nullptr, 0, 0, i1, i2, z, x, y, zz, tt, A.params, rr);
#pragma unroll
        for (int k = 0; k < XS_NRED; ++k) {
          acc[2 * k] += (double)rr[k].re;
          acc[2 * k + 1] += (double)rr[k].im;
        }
#endif
#if XS_NOUT_SITE > 0
        cx o[XS_NOUT_SITE];
        xs_obs_site(a, a, (const cx*)nullptr, (const cx*)nullptr, 0, 0, (const cx*)nullptr, x, y, zz, i1, i2, z, tt,
                    A.params, o);
#pragma unroll
        for (int k = 0; k < XS_NOUT_SITE; ++k) {
          sr[k][j] += (double)o[k].re;
          if (xs_ocplx_site(k)) si[k][j] += (double)o[k].im;
        }
#endif
      }
    }
#if XS_NRED > 0
    {
      const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
      for (int k = 0; k < 2 * XS_NRED; ++k) {
        const double s = xs_warp_sum(acc[k]);
        if (lane == 0) wred[warp][k] = s;
      }
      __syncthreads();
      if (tid < XS_NRED) {
        double re = 0, im = 0;
        for (int q = 0; q < 8; ++q) {
          re += wred[q][2 * tid];
          im += wred[q][2 * tid + 1];
        }
        A.redpart[((size_t)e * XS3_N3 + z) * XS_NRED + tid] = make_double2(re, im);
      }
    }
#endif
    __syncthreads();  // the plane buffer (and wred) are reused by the next trajectory
  }
  if (bad) atomicOr(A.status, 1);  // a diverged trajectory is reported at every observation
#if XS_NOUT_SITE > 0
  const double inv = 1.0 / (double)A.ens1;
  double2* out = gridDim.z == 1 ? A.av + ((size_t)b * A.npoints + A.n) * XS_OBS_STRIDE
                                : A.opart + ((size_t)blockIdx.z * gridDim.y + b) * ((size_t)XS_NOUT_SITE * XS_NS);
  const double sc = gridDim.z == 1 ? inv : 1.0;
#pragma unroll
  for (int k = 0; k < XS_NOUT_SITE; ++k)
#pragma unroll
    for (int j = 0; j < XS3_J; ++j) {
      const int i = tid + 256 * j;
      if (XS3_NP % 256 == 0 || i < XS3_NP)
        out[(size_t)k * XS_NS + (size_t)XS3_NP * z + i] = make_double2(sr[k][j] * sc, si[k][j] * sc);
    }
#endif
}

// Scalar observables from the per-trajectory reductions of the planes.
extern "C" __global__ void __launch_bounds__(256) xs_stream_scalar(const XsStreamArgs A) { xs_scalar_body<XS_NRG>(A); }
