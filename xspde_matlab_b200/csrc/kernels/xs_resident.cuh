// Resident-path kernel: every trajectory's field lives in shared memory for the
// whole time loop of one xpath call (Simulator/xpath.m:29-86).  One CTA owns
// XS_G trajectories of one ensemble block; the time loop, noise draws
// (Simulator/xnoise.m:29-38), interaction-picture steps (Applications/SDE/*.m,
// Applications/SPDE/xprop.m) and observables (Simulator/xdata.m:30-84) run
// on chip.  HBM sees only the initial/final fields and one partial-sum row of
// observables per output time.  Transforms along each space dimension are
// dense N x N matrices (FFT, DST-I/II/III, DCT-I/II/III alike), applied from
// L1/L2-resident tables; the propagator table exp(L dt) is FP64.
#pragma once

struct XsPathArgs {
  int ntraj;          // trajectories in this launch (multiple of XS_G)
  int ens1;           // trajectories per ensemble block
  int block0;         // global block index of the first trajectory
  int nc;             // 1 = fine pass, 2 = coarse pass
  int checks;         // p.checks(1)
  int npoints;        // p.points(1)
  int steps;          // p.steps(1)
  int seq;            // sequence index (Philox counter)
  u32 seed;
  int pad0;
  double wscale;      // sqrt(nscale * noisefactor)
  double vscale;      // sqrt(noisefactor)
  double dtr;         // step of this pass
  double t0;          // origin
  const double2* prop;  // [XS_PROP_COMPS][XS_NS] exp(L dtr / ipsteps)
  const cx* tmat;       // dense transforms, see xs_transform_dim
  int tmat_off[4];      // per space dim (index 1..3), element offsets
  const double2* a_in;  // optional [ntraj][F][NS] initial field (FP64)
  double2* a_out;       // optional [ntraj][F][NS] final field (FP64)
  double2* obs;         // [npoints][nctas][XS_OBS_STRIDE] observable partial sums
  int* status;          // bit 0: non-finite field
  int single_step;      // 1: one method step from t0 with the noise w_in (p.method)
  int pad1;
  const double* w_in;   // [NW, space, ens1] pre-scaled noise for single_step (null: zero)
  const double* params; // runtime named scalars p.<name> (prm[k])
  cx* gfield;           // XS_GFIELD: per-CTA field + scratch slices [grid][XS_NARR][G*F*NS]
  const double2* prop2; // exp(2 L dtr / ipsteps): two consecutive half-step propagators of MP
  const double2* bval;  // XS_BVAL: p.boundfun values [bval_n][ND][F][2] at t0 + k dtr/2
  const double2* bda;   // XS_BVAL: [ND][F] the da term of the Neumann patch (xpropfactor.m:45-50)
  int bval_n;
  int pad3;
  cx* aft;              // XS_SPEC: per trajectory tile [nt + npoints][G*F*NS]: the field at every
                        // step count, then its spectrum at the output frequencies
  const double2* twt;   // XS_SPEC: exp(2 pi i k / nt), k < nt
  int nt;               // XS_SPEC: points(1) x steps(1)
  int pad4;
  double fscn;          // XS_SPEC: p.fsc / nt
  double2* raw;         // optional raw trajectories (p.rawdata, xpath.m:73-78): the field at every
                        // output time in MATLAB's layout [F][npoints][NS][ntraj], fastest first
  const double2* kfilt; // XS_NK: [NK][NS] factors of p.nfilter on the FFT-ordered k lattice (null: 1)
  const double2* rfilt; // XS_NKV: the same for p.rfilter
  double kwscale;       // sqrt(nscale * knoisefactor), knoisefactor = prod(space points) / dv
  double kvscale;       // sqrt(knoisefactor)
};

// XS_GFIELD: the lattice is too large for shared memory, so each CTA keeps its
// field and transform scratch in its own slice of device memory (sized by the
// host so that the slices of all resident CTAs stay in L2 where possible) and
// only the reduction scratch in shared memory.  The code is the same; only the
// arrays' home differs (__syncthreads orders global accesses within a CTA).
#define XS_FARR (XS_GFIELD ? 0 : XS_NARR)
// XS_GFIELD: shared-memory copy of a real transform matrix (XS_MSM reals, 16-byte padded) ahead
// of the two tiles
#define XS_MS_CX ((((size_t)XS_MSM * sizeof(real) + 15) / 16) * 16 / sizeof(cx))
#define XS_NOMERGE (XS_BVAL || XS_SPEC)
// complex elements of one CTA's slice: the field arrays, then (methods other
// than MP) the two noise arrays of reals
#define XS_GSLICE ((size_t)(XS_NARR + XS_KARR + XS_KNARR) * XS_G * XS_F * XS_NS + (size_t)XS_WARR * XS_G * XS_NWS * XS_NS * sizeof(real) / sizeof(cx))

extern __shared__ __align__(16) unsigned char xs_smem[];

// k-filtered noise arrays (XS_KNARR field-sized complex arrays after the field
// arrays): ceil(NK/F) chunks of the current draw, as many of the first coarse
// draw, then ceil(NKV/F) chunks of the k-filtered randoms.  Component k of
// trajectory g at site s is element (k / F) G F NS + (g F + k % F) NS + s.
__device__ __forceinline__ cx* xs_zbuf(const XsPathArgs& P) {
  constexpr size_t GF = (size_t)XS_G * XS_F * XS_NS;
#if XS_GFIELD
  return P.gfield + (size_t)blockIdx.x * XS_GSLICE + (XS_NARR + XS_KARR) * GF;
#else
  (void)P;
  return (cx*)xs_smem + (XS_NARR + XS_KARR) * GF;
#endif
}
#define XS_ZIDX(k, g, s) ((size_t)((k) / XS_F) * (XS_G * XS_F * XS_NS) + ((g) * XS_F + (k) % XS_F) * XS_NS + (s))
// auxiliary cell (p.define): XS_NAC chunks after the k-filtered arrays, indexed like XS_ZIDX
__device__ __forceinline__ cx* xs_abuf(const XsPathArgs& P) {
  return xs_zbuf(P) + (size_t)(2 * XS_NKC + XS_NKVC) * XS_G * XS_F * XS_NS;
}
// one row of the time-spectrum record: the field, then the auxiliary chunks
#define XS_SPROW ((size_t)(1 + XS_NAC) * XS_G * XS_F * XS_NS)

#define XS_STRIDE1 1
#define XS_STRIDE2 (XS_N1)
#define XS_STRIDE3 (XS_N1 * XS_N2)

__device__ __forceinline__ void xs_site(int s, int& i1, int& i2, int& i3, real& x, real& y, real& z) {
  i1 = s % XS_N1;
  i2 = (s / XS_N1) % XS_N2;
  i3 = s / (XS_N1 * XS_N2);
  x = (real)(XS_O1 + XS_DX1 * (double)i1);
  y = (real)(XS_O2 + XS_DX2 * (double)i2);
  z = (real)(XS_O3 + XS_DX3 * (double)i3);
}

template <int D>
__device__ __forceinline__ void xs_transform_dim(cx* X, cx* T, const XsPathArgs& P, int dir) {
  constexpr int ND = D == 1 ? XS_N1 : (D == 2 ? XS_N2 : XS_N3);
  constexpr int SD = D == 1 ? XS_STRIDE1 : (D == 2 ? XS_STRIDE2 : XS_STRIDE3);
  if (ND <= 1) return;
  const cx* M0 = P.tmat + P.tmat_off[D];
  __syncthreads();
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) {
    const int s = i % XS_NS;
    const int gf = i / XS_NS;
    const int f = gf % XS_F;
    const int k = (s / SD) % ND;
    const int base = gf * XS_NS + s - k * SD;
    const cx* M = M0 + (size_t)(f * 2 + dir) * ND * ND;
    real ar = 0, ai = 0;
#pragma unroll 8
    for (int n = 0; n < ND; ++n) {
      const cx m = M[n * ND + k];
      const cx v = X[base + n * SD];
      ar += m.re * v.re - m.im * v.im;
      ai += m.re * v.im + m.im * v.re;
    }
    T[i] = mkcx(ar, ai);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) X[i] = T[i];
  __syncthreads();
}

// ---- shared-memory FFT for periodic power-of-two dimensions -----------------
// Stockham autosort FFT (Govindaraju et al., "High performance discrete Fourier
// transforms on graphics processors", SC 2008): stage with radix R after
// earlier stages of total radix NSP maps butterfly j (k = j mod NSP) as
//   v[r] = in[j + r N/R] * exp(-2 pi i k r / (NSP R)),  v = DFT_R(v),
//   out[(j / NSP) NSP R + k + r NSP] = v[r],
// ping-ponging between X and T; the output is in natural (MATLAB fft) order.
// The inverse is conj(FFT(conj(x))) / N, folded into the first load and the
// last store.  Twiddles exp(-2 pi i m / N) come from an FP64-built table.
template <int R> __device__ __forceinline__ void xs_dft_r(cx (&v)[R]);
template <> __device__ __forceinline__ void xs_dft_r<2>(cx (&v)[2]) {
  const cx a = v[0];
  v[0] = a + v[1];
  v[1] = a - v[1];
}
template <> __device__ __forceinline__ void xs_dft_r<4>(cx (&v)[4]) {
  const cx s02 = v[0] + v[2], d02 = v[0] - v[2], s13 = v[1] + v[3], d13 = v[1] - v[3];
  v[0] = s02 + s13;
  v[2] = s02 - s13;
  v[1] = mkcx(d02.re + d13.im, d02.im - d13.re);  // d02 - i d13
  v[3] = mkcx(d02.re - d13.im, d02.im + d13.re);  // d02 + i d13
}
template <> __device__ __forceinline__ void xs_dft_r<8>(cx (&v)[8]) {
  cx e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  xs_dft_r<4>(e);
  xs_dft_r<4>(o);
  const real c = (real)0.70710678118654752440;
  const cx t1 = mkcx(c * (o[1].re + o[1].im), c * (o[1].im - o[1].re));   // o1 exp(-i pi/4)
  const cx t2 = mkcx(o[2].im, -o[2].re);                                  // o2 (-i)
  const cx t3 = mkcx(c * (o[3].im - o[3].re), -c * (o[3].re + o[3].im));  // o3 exp(-3i pi/4)
  v[0] = e[0] + o[0];
  v[4] = e[0] - o[0];
  v[1] = e[1] + t1;
  v[5] = e[1] - t1;
  v[2] = e[2] + t2;
  v[6] = e[2] - t2;
  v[3] = e[3] + t3;
  v[7] = e[3] - t3;
}

// One stage along a dimension of length ND and site stride SD, over every
// line of every (trajectory, component) of the CTA.
template <int ND, int SD, int R, int NSP, bool FIRST, bool LAST>
__device__ __forceinline__ void xs_fft_stage(const cx* __restrict__ in, cx* __restrict__ out, const cx* __restrict__ tw,
                                             int inv) {
  constexpr int NB = ND / R;
  constexpr int NHI = XS_G * XS_F * XS_NS / (SD * ND);
  const real sc = (LAST ? (real)(1.0 / ND) : (real)1);
  for (int b = threadIdx.x; b < NHI * NB * SD; b += blockDim.x) {
    const int lo = b % SD, rem = b / SD;
    const int j = rem % NB, hi = rem / NB;
    const int base = lo + SD * ND * hi;
    const int k = j % NSP;
    cx v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      cx a = in[base + SD * (j + r * NB)];
      if (FIRST && inv) a.im = -a.im;
      if (NSP > 1 && r > 0) a = a * tw[k * r * (ND / (NSP * R))];
      v[r] = a;
    }
    xs_dft_r<R>(v);
    const int o0 = base + SD * ((j / NSP) * NSP * R + k);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      cx a = v[r];
      if (LAST && inv) a = mkcx(a.re * sc, -a.im * sc);
      out[o0 + SD * r * NSP] = a;
    }
  }
}

// Per-dimension stage sequences generated for the problem's lattice
// (specialisations of xs_fft_d for the dimensions flagged XS_FFTD<D>).
template <int D> __device__ __forceinline__ void xs_fft_d(cx*, cx*, const cx*, int) {}
XS_FFT_STAGES

#if XS_BVAL
// Boundary values of p.boundfun at time tb (host table at half steps t0 + k dtr/2).
__device__ __forceinline__ const double2* xs_bv(const XsPathArgs& P, double tb) {
  int k = (int)llrint((tb - P.t0) / (0.5 * P.dtr));
  k = k < 0 ? 0 : (k >= P.bval_n ? P.bval_n - 1 : k);
  return P.bval + (size_t)k * (XS_ND * XS_F * 2);
}
#endif

// xsetbound (Applications/SPDE/xsetbound.m:30-63): Dirichlet ends take the
// boundary values at time tb (zero without p.boundfun values).
__device__ __forceinline__ void xs_setbound(cx* X, const XsPathArgs* P = nullptr, double tb = 0) {
#if XS_SETBOUND
#if XS_BVAL
  if (!P) return;
  const double2* bv = xs_bv(*P, tb);
#else
  (void)P;
  (void)tb;
#endif
  for (int i = threadIdx.x; i < XS_G * XS_NS; i += blockDim.x) {
    const int g = i / XS_NS, s = i % XS_NS;
    int i1, i2, i3;
    real x, y, z;
    xs_site(s, i1, i2, i3, x, y, z);
#pragma unroll
    for (int f = 0; f < XS_F; ++f) {
#if XS_BVAL
      cx v;
      if (xs_dirichlet_val(f, i1, i2, i3, bv, v)) X[(g * XS_F + f) * XS_NS + s] = v;
#else
      if (xs_dirichlet(f, i1, i2, i3)) X[(g * XS_F + f) * XS_NS + s] = mkcx((real)0, (real)0);
#endif
    }
  }
  __syncthreads();
#endif
}

// ---- tiled line transforms (field in device memory) --------------------------
// A tile of TL lines along dimension D is loaded once into shared memory as
// S[n][l] (element n of line l, row stride LSP = padded TL), transformed there
// (Stockham stages ping-ponging S and S2, or the dense matrix into S2), and
// stored once: one read and one write of the field per transformed dimension.
template <int ND, int R, int NSP, bool FIRST, bool LAST, int TL, int LSP>
__device__ __forceinline__ void xs_fft_tstage(const cx* __restrict__ in, cx* __restrict__ out,
                                              const cx* __restrict__ tw, int inv) {
  constexpr int NB = ND / R;
  const real sc = (LAST ? (real)(1.0 / ND) : (real)1);
  for (int b = threadIdx.x; b < NB * TL; b += blockDim.x) {
    const int l = b % TL, j = b / TL;
    const int k = j % NSP;
    cx v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      cx a = in[(j + r * NB) * LSP + l];
      if (FIRST && inv) a.im = -a.im;
      if (NSP > 1 && r > 0) a = a * tw[k * r * (ND / (NSP * R))];
      v[r] = a;
    }
    xs_dft_r<R>(v);
    const int o0 = (j / NSP) * NSP * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      cx a = v[r];
      if (LAST && inv) a = mkcx(a.re * sc, -a.im * sc);
      out[(o0 + r * NSP) * LSP + l] = a;
    }
  }
}

// Generated per-dimension tile stage lists (return the buffer with the result).
template <int D> __device__ __forceinline__ cx* xs_fft_tile_d(cx* S, cx*, const cx*, int) { return S; }
XS_FFT_TILE_STAGES

#if XS_GFIELD
// Asynchronous global -> shared copy of one complex element (cp.async, completion by group).
__device__ __forceinline__ void xs_cp_async(cx* dst, const cx* src) {
  const u32 d = (u32)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(cx) == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void xs_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void xs_cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// The tile after the current one is copied into a third buffer while the current one is
// transformed, so its loads overlap the transform.
template <int D>
__device__ void xs_tr_tiled(cx* X, const XsPathArgs& P, int dir) {
  constexpr int ND = D == 1 ? XS_N1 : (D == 2 ? XS_N2 : XS_N3);
  constexpr int SD = D == 1 ? XS_STRIDE1 : (D == 2 ? XS_STRIDE2 : XS_STRIDE3);
  constexpr int TL = D == 1 ? XS_TL1 : (D == 2 ? XS_TL2 : XS_TL3);
  constexpr int LSP = D == 1 ? XS_LSP1 : (D == 2 ? XS_LSP2 : XS_LSP3);
  constexpr bool fft = D == 1 ? XS_FFTD1 : (D == 2 ? XS_FFTD2 : XS_FFTD3);
  if constexpr (ND > 1) {
    constexpr int NHI = XS_G * XS_F * XS_NS / (SD * ND);  // line groups (g, f, slower dims)
    constexpr int NPER = XS_NS / (SD * ND);               // line groups per (g, f)
    constexpr int NT = SD == 1 ? NHI / TL : NHI * (SD / (SD == 1 ? 1 : TL));
    constexpr bool RM = D == 1 ? XS_REALM1 : (D == 2 ? XS_REALM2 : XS_REALM3);
    real* Ms = (real*)xs_smem;  // real matrix of the current component (RM)
    int ms_f = -1;
    cx* S = (cx*)xs_smem + XS_MS_CX;
    cx* S2 = S + XS_TILE_ELEMS;
    cx* SN = S2 + XS_TILE_ELEMS;  // the next tile, in flight while S is transformed
    auto fetch = [&](int tile, cx* dst) {
      int hi0, lo0;
      if constexpr (SD == 1) { hi0 = tile * TL; lo0 = 0; }
      else { hi0 = tile / (SD / TL); lo0 = (tile % (SD / TL)) * TL; }
      for (int i = threadIdx.x; i < TL * ND; i += blockDim.x) {
        int n, l;
        size_t gi;
        if constexpr (SD == 1) { l = i / ND; n = i % ND; gi = (size_t)(hi0 + l) * ND + n; }
        else { n = i / TL; l = i % TL; gi = (size_t)lo0 + l + (size_t)SD * (n + (size_t)ND * hi0); }
        xs_cp_async(dst + n * LSP + l, X + gi);
      }
      xs_cp_commit();
    };
    fetch(0, S);
    for (int tile = 0; tile < NT; ++tile) {
      int hi0, lo0;
      if constexpr (SD == 1) { hi0 = tile * TL; lo0 = 0; }
      else { hi0 = tile / (SD / TL); lo0 = (tile % (SD / TL)) * TL; }
      xs_cp_wait_all();  // this tile's copies (the only group in flight)
      __syncthreads();
      if (tile + 1 < NT) fetch(tile + 1, SN);
      cx* Rb;
      if constexpr (fft) {
        Rb = xs_fft_tile_d<D>(S, S2, P.tmat + P.tmat_off[D], dir);
      } else {
        const int f = (hi0 / NPER) % XS_F;
        const cx* __restrict__ M = P.tmat + P.tmat_off[D] + (size_t)(f * 2 + dir) * ND * ND;
        // register block: KB outputs k x LB lines per thread; real matrices
        // (every DST/DCT type) skip the imaginary part of M and are read from
        // a shared-memory copy, KB entries per vector load
        constexpr int KB = ND % 4 == 0 ? 4 : 1;
        constexpr int LB = (TL % 2 == 0 && (ND / KB) * (TL / 2) >= XS_THREADS) ? 2 : 1;  // every thread busy
        constexpr bool MSH = RM && (size_t)ND * ND <= (size_t)XS_MSM;
        if constexpr (MSH) {
          if (f != ms_f) {  // tiles of one component share its matrix (uniform branch)
            for (int i = threadIdx.x; i < ND * ND; i += blockDim.x) Ms[i] = M[i].re;
            ms_f = f;
            __syncthreads();
          }
        }
        // mirror-symmetric matrices (M[N-1-n][k] = (-1)^(k+p) M[n][k], XS_FOLD = 1 + p, checked on
        // the host): fold each line into u_n = x_n + x_{N-1-n} (kept at n) and v_n = x_n - x_{N-1-n}
        // (kept at N-1-n); outputs with k + p even sum u, the others v, over n < N/2
        constexpr int FOLDP = D == 1 ? XS_FOLD1 : (D == 2 ? XS_FOLD2 : XS_FOLD3);
        constexpr bool FOLD = MSH && KB == 4 && FOLDP > 0;
        constexpr int PAR = FOLDP > 1 ? 1 : 0;
        constexpr int NN = FOLD ? ND / 2 : ND;
        if constexpr (FOLD) {
          for (int i = threadIdx.x; i < (ND / 2) * TL; i += blockDim.x) {
            const int n = i / TL, l = i % TL;
            const cx a = S[n * LSP + l], b = S[(ND - 1 - n) * LSP + l];
            S[n * LSP + l] = a + b;
            S[(ND - 1 - n) * LSP + l] = a - b;
          }
          __syncthreads();
        }
        for (int i = threadIdx.x; i < (ND / KB) * (TL / LB); i += blockDim.x) {
          const int l0 = (i % (TL / LB)) * LB, k0 = (i / (TL / LB)) * KB;
          real ar[KB][LB], ai[KB][LB];
#pragma unroll
          for (int q = 0; q < KB; ++q)
#pragma unroll
            for (int j = 0; j < LB; ++j) ar[q][j] = ai[q][j] = 0;
#pragma unroll 4
          for (int n = 0; n < NN; ++n) {
            cx v[LB], m[KB], vd[LB];
#pragma unroll
            for (int j = 0; j < LB; ++j) v[j] = S[n * LSP + l0 + j];
#pragma unroll
            for (int j = 0; j < LB; ++j) vd[j] = FOLD ? S[(ND - 1 - n) * LSP + l0 + j] : v[j];
            if constexpr (MSH && KB == 4 && sizeof(real) == 4) {
              const float4 q4 = *reinterpret_cast<const float4*>(Ms + n * ND + k0);
              m[0] = mkcx((real)q4.x, (real)0);
              m[1] = mkcx((real)q4.y, (real)0);
              m[2] = mkcx((real)q4.z, (real)0);
              m[3] = mkcx((real)q4.w, (real)0);
            } else if constexpr (MSH) {
#pragma unroll
              for (int q = 0; q < KB; ++q) m[q] = mkcx(Ms[n * ND + k0 + q], (real)0);
            } else {
#pragma unroll
              for (int q = 0; q < KB; ++q) m[q] = M[n * ND + k0 + q];
            }
#pragma unroll
            for (int q = 0; q < KB; ++q)
#pragma unroll
              for (int j = 0; j < LB; ++j) {
                const cx x = (FOLD && ((q + PAR) & 1)) ? vd[j] : v[j];  // k0 is a multiple of 4
                ar[q][j] += m[q].re * x.re;
                ai[q][j] += m[q].re * x.im;
                if (!RM) {
                  ar[q][j] -= m[q].im * v[j].im;
                  ai[q][j] += m[q].im * v[j].re;
                }
              }
          }
#pragma unroll
          for (int q = 0; q < KB; ++q)
#pragma unroll
            for (int j = 0; j < LB; ++j) S2[(k0 + q) * LSP + l0 + j] = mkcx(ar[q][j], ai[q][j]);
        }
        __syncthreads();
        Rb = S2;
      }
      for (int i = threadIdx.x; i < TL * ND; i += blockDim.x) {
        int n, l;
        size_t gi;
        if constexpr (SD == 1) { l = i / ND; n = i % ND; gi = (size_t)(hi0 + l) * ND + n; }
        else { n = i / TL; l = i % TL; gi = (size_t)lo0 + l + (size_t)SD * (n + (size_t)ND * hi0); }
        X[gi] = Rb[n * LSP + l];
      }
      __syncthreads();
      cx* const cur = S;
      S = SN;
      SN = cur;
    }
  }
}
#endif

// Transform along dimension D: generated Stockham stages (xs_fft_d<D>, defined
// by the problem header when XS_FFTD<D> is set) or the dense matrix.
template <int D>
__device__ __forceinline__ void xs_tr(cx* X, cx* T, const XsPathArgs& P, int dir) {
  constexpr bool fft = D == 1 ? XS_FFTD1 : (D == 2 ? XS_FFTD2 : XS_FFTD3);
#if XS_GFIELD
  if (true) {
    __syncthreads();
    xs_tr_tiled<D>(X, P, dir);
  } else
#endif
  if constexpr (fft) {
    __syncthreads();
    xs_fft_d<D>(X, T, P.tmat + P.tmat_off[D], dir);
    __syncthreads();
  } else {
    xs_transform_dim<D>(X, T, P, dir);
  }
}

// xprop (Applications/SPDE/xprop.m:18-42): transform, multiply by exp(L dt),
// inverse; with boundary values (XS_BVAL) the xpatch.m patch at time tb is
// taken off before and put back (with its Neumann term) after.
__device__ __forceinline__ void xs_prop_tab(cx* X, cx* T, const XsPathArgs& P, const double2* __restrict__ tab,
                                            double tb = 0) {
#if XS_HAS_PROP
#if XS_BVAL
  const double2* bv = xs_bv(P, tb);
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) {
    const int s = i % XS_NS, f = (i / XS_NS) % XS_F;
    int i1, i2, i3;
    real x, y, z;
    xs_site(s, i1, i2, i3, x, y, z);
    cx lp;
    X[i] = X[i] - xs_bpatch(f, i1, i2, i3, bv, P.bda, lp);
  }
  __syncthreads();
#else
  (void)tb;
#endif
  xs_tr<1>(X, T, P, 0);
  xs_tr<2>(X, T, P, 0);
  xs_tr<3>(X, T, P, 0);
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) {
    const int s = i % XS_NS;
    const int f = (i / XS_NS) % XS_F;
    const double2 pr = tab[(XS_PROP_COMPS > 1 ? f : 0) * XS_NS + s];
    const cx v = X[i];
    const double vr = (double)v.re, vi = (double)v.im;
    X[i] = mkcx((real)(vr * pr.x - vi * pr.y), (real)(vr * pr.y + vi * pr.x));
  }
  xs_tr<1>(X, T, P, 1);
  xs_tr<2>(X, T, P, 1);
  xs_tr<3>(X, T, P, 1);
#if XS_BVAL
  __syncthreads();
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) {
    const int s = i % XS_NS, f = (i / XS_NS) % XS_F;
    int i1, i2, i3;
    real x, y, z;
    xs_site(s, i1, i2, i3, x, y, z);
    cx lp;
    const cx pa = xs_bpatch(f, i1, i2, i3, bv, P.bda, lp);
    X[i] = X[i] + (pa + lp);
  }
#endif
#endif
  __syncthreads();
  xs_setbound(X, &P, tb);
  __syncthreads();
}
__device__ __forceinline__ void xs_prop(cx* X, cx* T, const XsPathArgs& P, double tb = 0) {
  xs_prop_tab(X, T, P, P.prop, tb);
}

#if XS_NK > 0 || XS_NKV > 0
// k-filtered Gaussian cell (Simulator/xnoise.m:40-46, xrandom.m:24-29): real
// standard normals on the FFT-ordered k lattice from the k stream, times the
// FP64 filter factor and the scale, then the inverse DFT along every space
// dimension (Applications/SPDE/xift.m) with the field's own transforms, one
// field-sized chunk at a time.
template <int NC>
__device__ void xs_kgen(cx* X, cx* T, const XsPathArgs& P, const double2* filt, int g0, int draw, double scale) {
  constexpr int GF = XS_G * XS_F * XS_NS;
  constexpr int NCH = (NC + XS_F - 1) / XS_F;
  __syncthreads();
  for (int i = threadIdx.x; i < NCH * GF; i += blockDim.x) {
    const int ch = i / GF, r = i - ch * GF;
    const int s = r % XS_NS, gf = r / XS_NS;
    const int f = gf % XS_F, g = gf / XS_F;
    const int k = ch * XS_F + f;
    cx v = mkcx((real)0, (real)0);
    if (k < NC) {
      const int e = g0 + g;
      const double zr = (double)xs_knormal(k, (u32)s, (u32)(e % P.ens1), (u32)draw, (u32)P.seq, P.seed,
                                           (u32)(P.block0 + e / P.ens1));
      const double2 fv = filt ? filt[(size_t)k * XS_NS + s] : make_double2(1.0, 0.0);
      v = mkcx((real)(zr * fv.x * scale), (real)(zr * fv.y * scale));
    }
    X[i] = v;
  }
  __syncthreads();
  for (int ch = 0; ch < NCH; ++ch) {
    cx* C = X + (size_t)ch * GF;
    xs_tr<1>(C, T, P, 1);
    xs_tr<2>(C, T, P, 1);
    xs_tr<3>(C, T, P, 1);
  }
  __syncthreads();
}
#endif

// k-filtered noise of one p.noisegen call (xnoise.m:39-50): mode 0 fine draw,
// 1 first coarse draw (kept), 2 second coarse draw averaged with the first.
__device__ __forceinline__ void xs_knoise(const XsPathArgs& P, cx* T, int mode, int draw, int g0) {
#if XS_NK > 0
  constexpr size_t GF = (size_t)XS_G * XS_F * XS_NS;
  cx* Z = xs_zbuf(P);
  cx* Zp = Z + XS_NKC * GF;
  xs_kgen<XS_NK>(mode == 1 ? Zp : Z, T, P, P.kfilt, g0, draw, P.kwscale);
  if (mode == 2) {
    for (size_t i = threadIdx.x; i < XS_NKC * GF; i += blockDim.x) Z[i] = (Z[i] + Zp[i]) * (real)0.5;
    __syncthreads();
  }
#else
  (void)P; (void)T; (void)mode; (void)draw; (void)g0;
#endif
}

#if XS_NA > 0
// Auxiliary cell (Simulator/xpath.m:36-45): X = define(A, w, t), or with `avg` the
// mean of X and define(A, w, t) (the method sits between the two evaluations,
// with the same noise and the same p.t).
__device__ void xs_aux(const cx* A, cx* X, const real* W, const cx* Z, double t, const XsPathArgs& P, bool avg) {
  __syncthreads();
  for (int i = threadIdx.x; i < XS_G * XS_NS; i += blockDim.x) {
    const int g = i / XS_NS, s = i % XS_NS;
    int i1, i2, i3;
    real x, y, z;
    xs_site(s, i1, i2, i3, x, y, z);
    cx a[XS_F], o[XS_NA];
    real w[XS_NWS];
    cx zk[XS_NK > 0 ? XS_NK : 1];
#pragma unroll
    for (int f = 0; f < XS_F; ++f) a[f] = A[(g * XS_F + f) * XS_NS + s];
#pragma unroll
    for (int c = 0; c < XS_NWS; ++c) w[c] = XS_NW > 0 ? W[(g * XS_NWS + c) * XS_NS + s] : (real)0;
#pragma unroll
    for (int k = 0; k < XS_NK; ++k) zk[k] = Z[XS_ZIDX(k, g, s)];
    (void)Z;
    xs_define(a, w, zk, x, y, z, (real)t, P.params, A, g, s, o);
#pragma unroll
    for (int k = 0; k < XS_NA; ++k) {
      cx& d = X[XS_ZIDX(k, g, s)];
      d = avg ? (d + o[k]) * (real)0.5 : o[k];
    }
  }
  __syncthreads();
}
#endif

// dst = base + h * deriv(src, w, t), pointwise over sites (all components at once).
// dst = base + h * deriv(src, w, t).  A drift with finite differences
// (XS_STENCIL) reads neighbours of src, so an in-place update (dst == src)
// writes through the transform scratch T first.
__device__ __forceinline__ void xs_deriv_update(cx* dst, const cx* base, const cx* src, const real* W, const cx* Z,
                                                real h, double t, const double* prm, cx* T) {
  cx* out = (XS_STENCIL && dst == src) ? T : dst;
  for (int i = threadIdx.x; i < XS_G * XS_NS; i += blockDim.x) {
    const int g = i / XS_NS, s = i % XS_NS;
    int i1, i2, i3;
    real x, y, z;
    xs_site(s, i1, i2, i3, x, y, z);
    cx a[XS_F], d[XS_F];
    real w[XS_NW > 0 ? XS_NW : 1];
#pragma unroll
    for (int f = 0; f < XS_F; ++f) a[f] = src[(g * XS_F + f) * XS_NS + s];
#pragma unroll
    for (int c = 0; c < XS_NW; ++c) w[c] = W[(g * XS_NWS + c) * XS_NS + s];
    cx zk[XS_NK > 0 ? XS_NK : 1];
#pragma unroll
    for (int k = 0; k < XS_NK; ++k) zk[k] = Z[XS_ZIDX(k, g, s)];
    (void)Z;
    xs_deriv(a, w, zk, x, y, z, (real)t, prm, src, g, s, d);
#pragma unroll
    for (int f = 0; f < XS_F; ++f) {
      const int j = (g * XS_F + f) * XS_NS + s;
      out[j] = base[j] + h * d[f];
    }
  }
  __syncthreads();
  if (out != dst) {
    for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) dst[i] = out[i];
    __syncthreads();
  }
}

__device__ __forceinline__ void xs_axpby(cx* dst, real ca, const cx* A, real cb, const cx* B) {
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) dst[i] = ca * A[i] + cb * B[i];
  __syncthreads();
}
__device__ __forceinline__ void xs_copy(cx* dst, const cx* src) {
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// One interaction-picture step of the selected method.  t is the time at the
// start of the step (xpath's p.t).
__device__ void xs_method(cx* A, cx* B1, cx* B2, cx* B3, cx* T, const real* W, const XsPathArgs& P, double t) {
  const double dtr = P.dtr;
  const cx* Z = xs_zbuf(P);
  (void)Z;
#if XS_METHOD == 0
  // MP (Applications/SDE/MP.m:10-27)
  const real h = (real)(dtr * 0.5);
  xs_prop(A, T, P, t);
  xs_copy(B1, A);
  for (int it = 0; it < XS_ITER; ++it) {
    xs_deriv_update(A, B1, A, W, Z, h, t + dtr * 0.5, P.params, T);
    xs_setbound(A, &P, t + dtr * 0.5);
  }
  xs_axpby(A, (real)2, A, (real)-1, B1);
  xs_prop(A, T, P, t + dtr);
#elif XS_METHOD == 1
  // RK4 (Applications/SDE/RK4.m:7-42)
  const real h = (real)(dtr * 0.5);
  xs_setbound(A);
  xs_deriv_update(B1, A, A, W, Z, h, t, P.params, T);
  xs_prop(B1, T, P);
  xs_prop(A, T, P);
  xs_deriv_update(B2, A, B1, W, Z, h, t + dtr * 0.5, P.params, T);
  xs_setbound(B2);
  xs_deriv_update(B3, A, B2, W, Z, (real)(2 * (dtr * 0.5)), t + dtr * 0.5, P.params, T);
  xs_setbound(B3);
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x)
    A[i] = (B1[i] + (real)2 * B2[i] + B3[i] - A[i]) / (real)3;
  __syncthreads();
  xs_prop(A, T, P);
  xs_prop(B3, T, P);
  xs_deriv_update(A, A, B3, W, Z, (real)(dtr * 0.5 / 3.0), t + dtr, P.params, T);
  xs_setbound(A);
#elif XS_METHOD == 2
  // Euler (Applications/SDE/Euler.m:6-10)
  xs_deriv_update(A, A, A, W, Z, (real)dtr, t, P.params, T);
  xs_prop(A, T, P);
#elif XS_METHOD == 3
  // RK2 (Applications/SDE/RK2.m:7-25): B1 holds the predictor a.
  xs_deriv_update(B1, A, A, W, Z, (real)dtr, t, P.params, T);
  xs_prop(A, T, P);
  xs_prop(B1, T, P);
  xs_deriv_update(A, A, B1, W, Z, (real)dtr, t + dtr, P.params, T);
  xs_axpby(A, (real)0.5, B1, (real)0.5, A);
#elif XS_METHOD == 4
  // Implicit (Applications/SDE/Implicit.m:8-17)
  xs_copy(B1, A);
  for (int it = 0; it < XS_ITER; ++it) xs_deriv_update(A, B1, A, W, Z, (real)dtr, t + dtr, P.params, T);
  xs_prop(A, T, P);
#endif
  __syncthreads();
}

#if XS_LEAN
// MP step with the midpoint iterations fused per site (Applications/SDE/MP.m:
// 13-23): the iterations are pointwise, so a0, the iterate and the noise live
// in registers and only the field and the transform scratch stay in shared
// memory.  mode 0: fine draw `draw`; 2: coarse pass, mean of draws `prev` and
// `draw` (Simulator/xnoise.m:33-35); 3: the caller's noise P.w_in (p.method).
// The arithmetic is that of the unfused step, operation for operation.
// Consecutive half-step propagators of neighbouring steps are merged, as in
// the streaming path: `merged` = the previous step's second half is still
// pending, so the first half applies exp(2 L dt/2) (P.prop2); with `last` the
// step ends with its own second half, otherwise that half is left pending.
__device__ void xs_mp_lean(cx* A, cx* T, const XsPathArgs& P, double t, int g0, int mode, int draw, int prev,
                           bool merged, bool last) {
  const double dtr = P.dtr;
  const real h = (real)(dtr * 0.5);
  const real tm = (real)(t + dtr * 0.5);
  xs_prop_tab(A, T, P, merged ? P.prop2 : P.prop, t);
#if XS_BVAL
  const double2* bvm = xs_bv(P, t + dtr * 0.5);  // Dirichlet values during the midpoint iterations
#endif
  for (int i = threadIdx.x; i < XS_G * XS_NS; i += blockDim.x) {
    const int g = i / XS_NS, s = i % XS_NS;
    const int e = g0 + g;
    int i1, i2, i3;
    real x, y, z;
    xs_site(s, i1, i2, i3, x, y, z);
    real w[XS_NWS];
#if XS_NW > 0
    if (mode == 3) {
#pragma unroll
      for (int c = 0; c < XS_NW; ++c)
        w[c] = P.w_in ? (real)P.w_in[c + (size_t)XS_NW * (s + (size_t)XS_NS * e)] : (real)0;
    } else {
      const u32 blk = (u32)(P.block0 + e / P.ens1);
      const u32 el = (u32)(e % P.ens1);
      real zz[XS_NW];
      xs_normals_site<XS_NW>(zz, (u32)s, el, (u32)draw, (u32)P.seq, P.seed, blk);
#pragma unroll
      for (int c = 0; c < XS_NW; ++c) w[c] = xs_mul_rn(zz[c], (real)P.wscale);
      if (mode == 2) {
        xs_normals_site<XS_NW>(zz, (u32)s, el, (u32)prev, (u32)P.seq, P.seed, blk);
#pragma unroll
        for (int c = 0; c < XS_NW; ++c) w[c] = (w[c] + xs_mul_rn(zz[c], (real)P.wscale)) * (real)0.5;
      }
    }
#else
    w[0] = (real)0;
#endif
    cx zk[XS_NK > 0 ? XS_NK : 1];
#if XS_NK > 0
    {
      const cx* Z = xs_zbuf(P);
#pragma unroll
      for (int k = 0; k < XS_NK; ++k) zk[k] = Z[XS_ZIDX(k, g, s)];
    }
#endif
    cx a0[XS_F], a[XS_F], d[XS_F];
#pragma unroll
    for (int f = 0; f < XS_F; ++f) a0[f] = a[f] = A[(g * XS_F + f) * XS_NS + s];
    for (int it = 0; it < XS_ITER; ++it) {
      xs_deriv(a, w, zk, x, y, z, tm, P.params, A, g, s, d);
#pragma unroll
      for (int f = 0; f < XS_F; ++f) {
        a[f] = a0[f] + h * d[f];
#if XS_SETBOUND
#if XS_BVAL
        {
          cx bvv;
          if (xs_dirichlet_val(f, i1, i2, i3, bvm, bvv)) a[f] = bvv;
        }
#else
        if (xs_dirichlet(f, i1, i2, i3)) a[f] = mkcx((real)0, (real)0);
#endif
#endif
      }
    }
#pragma unroll
    for (int f = 0; f < XS_F; ++f) A[(g * XS_F + f) * XS_NS + s] = (real)2 * a[f] - a0[f];
  }
  __syncthreads();
  if (last) xs_prop(A, T, P, t + dtr);
  __syncthreads();
}
#endif

// Noise of one p.noisegen call into W (coarse pass: averaged with Wp, xnoise.m:33-35).
__device__ __forceinline__ void xs_noise(real* W, real* Wp, int mode, int draw, int g0, const XsPathArgs& P) {
#if XS_NW > 0
  for (int i = threadIdx.x; i < XS_G * XS_NS; i += blockDim.x) {
    const int g = i / XS_NS, s = i % XS_NS;
    const int e = g0 + g;
    const u32 blk = (u32)(P.block0 + e / P.ens1);
    const u32 el = (u32)(e % P.ens1);
    real z[XS_NW];
    xs_normals_site<XS_NW>(z, (u32)s, el, (u32)draw, (u32)P.seq, P.seed, blk);
#pragma unroll
    for (int c = 0; c < XS_NW; ++c) {
      const int j = (g * XS_NWS + c) * XS_NS + s;
      const real v = xs_mul_rn(z[c], (real)P.wscale);
      if (mode == 0) W[j] = v;                          // fine draw
      else if (mode == 1) Wp[j] = v;                    // first coarse draw
      else W[j] = (v + Wp[j]) * (real)0.5;              // averaged coarse draw
    }
  }
  __syncthreads();
#endif
}

// Observables at one output time: per-CTA sums over its trajectories.
// K (XS_KOBS): the field Fourier-transformed along the flagged dimensions for
// the observables with p.transforms (xnft.m: fft along each, times dx/sqrt(2 pi));
// T is the transform scratch, free at output times.
// phase 0 writes the slots of observables on the field at the output time, phase 1
// (XS_SPEC) those on its time spectrum; A is then the spectral field of output n.
__device__ void xs_observe(const cx* A, const cx* AX, cx* RED, int n, double t, const XsPathArgs& P, double* wsum,
                           int cta, int nctas, cx* K, cx* T, int phase) {
  (void)AX;
#define XS_LOAD_XA(g, s)                                                          \
  cx xa[XS_NA > 0 ? XS_NA : 1];                                                   \
  _Pragma("unroll") for (int k = 0; k < XS_NA; ++k) xa[k] = AX[XS_ZIDX(k, (g), (s))];
  double2* out = P.obs + ((size_t)n * nctas + cta) * XS_OBS_STRIDE;
#if XS_KOBS
  for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) K[i] = A[i];
  __syncthreads();
  if (XS_KTR1) xs_tr<1>(K, T, P, 0);
  if (XS_KTR2) xs_tr<2>(K, T, P, 0);
  if (XS_KTR3) xs_tr<3>(K, T, P, 0);
  __syncthreads();
#define XS_LOAD_AK(g, s)                                                          \
  _Pragma("unroll") for (int f = 0; f < XS_F; ++f) ak[f] = K[((g) * XS_F + f) * XS_NS + (s)] * (real)XS_KFACT;
#else
  (void)K;
  (void)T;
#define XS_LOAD_AK(g, s)                                                          \
  _Pragma("unroll") for (int f = 0; f < XS_F; ++f) ak[f] = a[f];
#endif
#if XS_NRED > 0
  // full-space reductions (Int/Ave) per trajectory
  for (int g = 0; g < XS_G; ++g) {
    double acc[2 * XS_NRED];
#pragma unroll
    for (int k = 0; k < 2 * XS_NRED; ++k) acc[k] = 0;
    for (int s = threadIdx.x; s < XS_NS; s += blockDim.x) {
      int i1, i2, i3;
      real x, y, z;
      xs_site(s, i1, i2, i3, x, y, z);
      cx a[XS_F], ak[XS_F], r[XS_NRED];
#pragma unroll
      for (int f = 0; f < XS_F; ++f) a[f] = A[(g * XS_F + f) * XS_NS + s];
      XS_LOAD_AK(g, s)
      XS_LOAD_XA(g, s)
      xs_integrands(a, ak, xa, A, g, s, i1, i2, i3, x, y, z, (real)t, P.params, r);
#pragma unroll
      for (int k = 0; k < XS_NRED; ++k) { acc[2 * k] += (double)r[k].re; acc[2 * k + 1] += (double)r[k].im; }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < 2 * XS_NRED; ++k) {
      double v = xs_warp_sum(acc[k]);
      if (lane == 0) wsum[warp * 2 * XS_NRED + k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 2 * XS_NRED) {
      double v = 0;
      for (int q = 0; q < nw; ++q) v += wsum[q * 2 * XS_NRED + threadIdx.x];
      real* rr = (real*)(RED + g * XS_NRED);
      rr[threadIdx.x] = (real)v;
    }
    __syncthreads();
  }
#endif
#if XS_NOUT_SITE > 0
  for (int s = threadIdx.x; s < XS_NS; s += blockDim.x) {
    int i1, i2, i3;
    real x, y, z;
    xs_site(s, i1, i2, i3, x, y, z);
    double sr[XS_NOUT_SITE], si[XS_NOUT_SITE], cr[XS_NOUT_SITE], ci[XS_NOUT_SITE];  // compensated sums
#pragma unroll
    for (int k = 0; k < XS_NOUT_SITE; ++k) sr[k] = si[k] = cr[k] = ci[k] = 0;
    for (int g = 0; g < XS_G; ++g) {
      cx a[XS_F], ak[XS_F], o[XS_NOUT_SITE];
#pragma unroll
      for (int f = 0; f < XS_F; ++f) a[f] = A[(g * XS_F + f) * XS_NS + s];
      XS_LOAD_AK(g, s)
      XS_LOAD_XA(g, s)
      xs_obs_site(a, ak, xa, A, g, s, RED + g * (XS_NRED > 0 ? XS_NRED : 1), x, y, z, i1, i2, i3, (real)t, P.params, o);
#pragma unroll
      for (int k = 0; k < XS_NOUT_SITE; ++k) {
        xs_kadd(sr[k], cr[k], (double)o[k].re);
        if (xs_ocplx_site(k)) xs_kadd(si[k], ci[k], (double)o[k].im);
      }
    }
#pragma unroll
    for (int k = 0; k < XS_NOUT_SITE; ++k)
      if (xs_ospec_site(k) == phase) out[(size_t)k * XS_NS + s] = make_double2(sr[k] + cr[k], si[k] + ci[k]);
  }
#endif
#if XS_NOUT_SCALAR > 0
  if (threadIdx.x == 0) {
    double sr[XS_NOUT_SCALAR], si[XS_NOUT_SCALAR], cr[XS_NOUT_SCALAR], ci[XS_NOUT_SCALAR];
    for (int k = 0; k < XS_NOUT_SCALAR; ++k) sr[k] = si[k] = cr[k] = ci[k] = 0;
    for (int g = 0; g < XS_G; ++g) {
      cx o[XS_NOUT_SCALAR];
      xs_obs_scalar(RED + g * (XS_NRED > 0 ? XS_NRED : 1), (real)t, P.params, o);
      for (int k = 0; k < XS_NOUT_SCALAR; ++k) {
        xs_kadd(sr[k], cr[k], (double)o[k].re);
        xs_kadd(si[k], ci[k], (double)o[k].im);
      }
    }
    for (int k = 0; k < XS_NOUT_SCALAR; ++k)
      if (xs_ospec_scalar(k) == phase)
        out[(size_t)XS_NOUT_SITE * XS_NS + k] = make_double2(sr[k] + cr[k], si[k] + ci[k]);
  }
#endif
#undef XS_LOAD_AK
#undef XS_LOAD_XA
  __syncthreads();
}

#if XS_SPEC
// Time spectrum (Simulator/xpath.m:46-68, 90-106).  Row n1 of the tile's record holds
// the field after step count n1 (the initial field at n1 = 0); the fine pass of a
// checked run stores the mean of its two half steps.
__device__ void xs_spec_store(const cx* A, const XsPathArgs& P, int cta, int n1, bool avg) {
  constexpr int GF = XS_G * XS_F * XS_NS;
  cx* S = P.aft + ((size_t)cta * (P.nt + P.npoints) + n1) * XS_SPROW;
  __syncthreads();
  for (int i = threadIdx.x; i < GF; i += blockDim.x) S[i] = avg ? (A[i] + S[i]) * (real)0.5 : A[i];
#if XS_NA > 0
  const cx* X = xs_abuf(P);
  for (size_t i = threadIdx.x; i < XS_SPROW - GF; i += blockDim.x)
    S[GF + i] = avg ? (X[i] + S[GF + i]) * (real)0.5 : X[i];
#endif
  __syncthreads();
}

// Spectral field of output n: fsc/nt sum_j a_j exp(2 pi i m j / nt), m = n - floor(P1/2)
// (ifft along time, fftshift, p.specpts), in FP64 from the FP64 table; each thread owns
// one site of one trajectory and forms XS_SPEC_NB frequencies per pass over the record.
#define XS_SPEC_NB 4
__device__ void xs_spectrum(const XsPathArgs& P, int cta) {
  constexpr size_t GF = XS_SPROW;  // field and auxiliary chunks
  const int nt = P.nt, np = P.npoints;
  cx* S = P.aft + (size_t)cta * (nt + np) * GF;
  __syncthreads();
  for (size_t i = threadIdx.x; i < GF; i += blockDim.x) {
    for (int n0 = 0; n0 < np; n0 += XS_SPEC_NB) {
      double re[XS_SPEC_NB], im[XS_SPEC_NB];
      int ph[XS_SPEC_NB], dm[XS_SPEC_NB];
#pragma unroll
      for (int b = 0; b < XS_SPEC_NB; ++b) {
        const int m = n0 + b - np / 2;
        dm[b] = ((m % nt) + nt) % nt;
        ph[b] = 0;
        re[b] = im[b] = 0;
      }
      for (int j = 0; j < nt; ++j) {
        const cx x = S[(size_t)j * GF + i];
        const double xr = (double)x.re, xi = (double)x.im;
#pragma unroll
        for (int b = 0; b < XS_SPEC_NB; ++b) {
          const double2 w = P.twt[ph[b]];
          re[b] += xr * w.x - xi * w.y;
          im[b] += xr * w.y + xi * w.x;
          ph[b] += dm[b];
          if (ph[b] >= nt) ph[b] -= nt;
        }
      }
#pragma unroll
      for (int b = 0; b < XS_SPEC_NB; ++b)
        if (n0 + b < np) S[(size_t)(nt + n0 + b) * GF + i] = mkcx((real)(re[b] * P.fscn), (real)(im[b] * P.fscn));
    }
  }
  __syncthreads();
}
#endif

// Shared-memory layout of one CTA (XS_SMEM_BYTES in total).  False, with
// status bit 1 set, when this launch's dynamic shared memory or block size do
// not match the layout; the CTA must then return without touching it.
__device__ __forceinline__ bool xs_layout_ok(int* status) {
  constexpr size_t GF = (size_t)XS_G * XS_F * XS_NS;
  constexpr size_t need = ((XS_GFIELD ? 0 : XS_NARR + XS_KARR + XS_KNARR) * GF + 3 * (size_t)XS_TILE_ELEMS + (XS_GFIELD ? XS_MS_CX : 0)) * sizeof(cx) + (size_t)XS_G * (XS_NRED > 0 ? XS_NRED : 1) * sizeof(cx) +
                          32 * 2 * (XS_NRED > 0 ? XS_NRED : 1) * sizeof(double) +
                          (XS_GFIELD ? 0 : XS_WARR) * (size_t)XS_G * XS_NWS * XS_NS * sizeof(real);
  u32 dyn;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
  if (need > (size_t)dyn || need != (size_t)XS_SMEM_BYTES || (int)blockDim.x != XS_THREADS) {
    if (threadIdx.x == 0) atomicOr(status, 2);
    return false;
  }
  return true;
}

// One CTA's share of an xpath call: trajectories cta*G .. cta*G+G-1 of P,
// observable partial sums in row `cta` of `nctas`.
__device__ void xs_resident_run(const XsPathArgs& P, int cta, int nctas) {
  constexpr int GF = XS_G * XS_F * XS_NS;
#if XS_GFIELD
  cx* A = P.gfield + (size_t)blockIdx.x * XS_GSLICE;
  cx* RED = (cx*)xs_smem + XS_MS_CX + 3 * XS_TILE_ELEMS;  // after the matrix copy and the three tiles; [G][NRED]
#else
  cx* A = (cx*)xs_smem;
  cx* RED = A + (XS_NARR + XS_KARR + XS_KNARR) * GF;  // [G][NRED]
#endif
  cx* K = A + XS_NARR * GF;  // k-space copy of the field (XS_KARR)
  cx* B1 = A + GF;
  cx* B2 = B1 + (XS_NARR >= 3 ? GF : 0);
  cx* B3 = B2 + (XS_NARR >= 4 ? GF : 0);
  cx* T = A + (XS_NARR - 1) * GF;     // transform scratch is the last array
  double* wsum = (double*)(RED + XS_G * (XS_NRED > 0 ? XS_NRED : 1));  // [32][2*NRED]
#if XS_GFIELD
  real* W = (real*)(A + (XS_NARR + XS_KARR + XS_KNARR) * GF);  // noise arrays follow the field arrays in the CTA's slice
#else
  real* W = (real*)(wsum + 32 * 2 * (XS_NRED > 0 ? XS_NRED : 1));
#endif
  real* Wp = W + XS_G * XS_NWS * XS_NS;
  const int g0 = cta * XS_G;
  if ((cta + 1) * XS_G > P.ntraj || cta >= nctas) {
    if (threadIdx.x == 0) atomicOr(P.status, 2);
    return;
  }

  // initial field: p.initial(v,p) with v = p.randomgen(p) (xensemble.m:53-64)
#if XS_NKV > 0
  cx* VK = xs_zbuf(P) + 2 * XS_NKC * GF;  // k-filtered randoms (xrandom.m:24-29), draw 0 of the k stream
  if (!P.a_in) xs_kgen<XS_NKV>(VK, T, P, P.rfilt, g0, 0, P.kvscale);
#endif
  for (int i = threadIdx.x; i < XS_G * XS_NS; i += blockDim.x) {
    const int g = i / XS_NS, s = i % XS_NS;
    const int e = g0 + g;
    cx a[XS_F];
    if (P.a_in) {
#pragma unroll
      for (int f = 0; f < XS_F; ++f) {
        const double2 v = P.a_in[((size_t)e * XS_F + f) * XS_NS + s];
        a[f] = mkcx((real)v.x, (real)v.y);
      }
    } else {
      int i1, i2, i3;
      real x, y, z;
      xs_site(s, i1, i2, i3, x, y, z);
      real v[XS_NV > 0 ? XS_NV : 1];
#if XS_NV > 0
      xs_normals_site<XS_NV>(v, (u32)s, (u32)(e % P.ens1), 0u, (u32)P.seq, P.seed, (u32)(P.block0 + e / P.ens1));
#pragma unroll
      for (int c = 0; c < XS_NV; ++c) v[c] *= (real)P.vscale;
#endif
      cx vk[XS_NKV > 0 ? XS_NKV : 1];
#if XS_NKV > 0
#pragma unroll
      for (int k = 0; k < XS_NKV; ++k) vk[k] = VK[XS_ZIDX(k, g, s)];
#endif
      xs_initial(v, vk, x, y, z, P.params, a);
    }
#pragma unroll
    for (int f = 0; f < XS_F; ++f) A[(g * XS_F + f) * XS_NS + s] = a[f];
  }
  __syncthreads();
#if XS_NA > 0
  // initial auxiliary cell (xensemble.m:74-77): p.define on a noise draw of its own (Philox draw
  // 2^32 - 1), at p.t = origin, or origin - 1 when boundary values were set before it (:67-72)
  cx* AUX = xs_abuf(P);
  if (!P.single_step) {
    xs_noise(W, Wp, 0, -1, g0, P);
    if (XS_NK > 0) xs_knoise(P, T, 0, -1, g0);
    xs_aux(A, AUX, W, xs_zbuf(P), P.t0 - ((XS_SETBOUND && XS_ND > 0) ? 1.0 : 0.0), P, false);
  }
#else
  const cx* AUX = nullptr;
#endif

  double t = P.t0;
  if (P.single_step) {
    // p.method(a, w, p) on the given noise (Simulator/xpath.m:42)
#if !XS_LEAN
    for (int i = threadIdx.x; i < XS_G * XS_NS; i += blockDim.x) {
      const int g = i / XS_NS, s = i % XS_NS;
      const size_t e = (size_t)(g0 + g);
#pragma unroll
      for (int c = 0; c < XS_NW; ++c)
        W[(g * XS_NWS + c) * XS_NS + s] = P.w_in ? (real)P.w_in[c + (size_t)XS_NW * (s + (size_t)XS_NS * e)] : (real)0;
    }
#endif
    __syncthreads();
#if XS_LEAN
    xs_mp_lean(A, T, P, P.t0, g0, 3, 0, 0, false, true);
#else
    xs_method(A, B1, B2, B3, T, W, P, P.t0);
#endif
  } else {
  int draw = 0;
  bool pending = false;  // lean MP: second half-step propagator not yet applied
  for (int n = 0; n < P.npoints; ++n) {
    for (int step = 0; step < P.steps; ++step) {
      if (n > 0 || step > 0 || P.npoints == 1) {
        for (int chk = 0; chk <= P.checks; ++chk) {
          ++draw;
          int mode = 0;
          if (P.nc == 2 && P.checks) mode = chk == 0 ? 1 : 2;
          if (XS_NK > 0) xs_knoise(P, T, mode, draw, g0);
#if XS_LEAN
          if (P.nc == 1 || chk == 1) {
            __syncthreads();
            // time-dependent boundary patches (XS_BVAL) and the spectrum record (XS_SPEC)
            // forbid merging half steps
            xs_mp_lean(A, T, P, t, g0, mode, draw, draw - 1, pending && !XS_NOMERGE, XS_NOMERGE != 0);
            pending = !XS_NOMERGE;
            t += P.dtr;
#if XS_SPEC
            xs_spec_store(A, P, cta, n * P.steps + step, P.nc == 1 && chk == 1);
#endif
          }
#else
          xs_noise(W, Wp, mode, draw, g0, P);
          if (P.nc == 1 || chk == 1) {
            __syncthreads();
#if XS_NA > 0
            xs_aux(A, AUX, W, xs_zbuf(P), t, P, false);  // xpath.m:36-38
#endif
            xs_method(A, B1, B2, B3, T, W, P, t);
#if XS_NA > 0
            xs_aux(A, AUX, W, xs_zbuf(P), t, P, true);   // xpath.m:42-44
#endif
            t += P.dtr;
#if XS_SPEC
            xs_spec_store(A, P, cta, n * P.steps + step, P.nc == 1 && chk == 1);
#endif
          }
#endif
        }
      }
#if XS_SPEC
      else {
        xs_spec_store(A, P, cta, 0, false);
      }
#endif
      if (step == 0) {
        __syncthreads();
#if XS_LEAN
        if (pending) xs_prop(A, T, P);
        pending = false;
#endif
        if (P.raw) {
          __syncthreads();
          for (int i = threadIdx.x; i < GF; i += blockDim.x) {
            const int g = i / (XS_F * XS_NS), f = (i / XS_NS) % XS_F, s = i % XS_NS;
            const cx v = A[i];
            P.raw[f + (size_t)XS_F * (n + (size_t)P.npoints * (s + (size_t)XS_NS * (g0 + g)))] =
                make_double2((double)v.re, (double)v.im);
          }
        }
        xs_observe(A, AUX, RED, n, t, P, wsum, cta, nctas, K, T, 0);
      }
    }
  }
#if XS_LEAN
  if (pending) xs_prop(A, T, P);
#endif
  }
  __syncthreads();
  // final field and non-finite check
  bool bad = false;
  for (int i = threadIdx.x; i < GF; i += blockDim.x) {
    const cx v = A[i];
    if (!isfinite((double)v.re) || !isfinite((double)v.im)) bad = true;
    if (P.a_out) {
      const int g = i / (XS_F * XS_NS);
      P.a_out[(size_t)(g0 + g) * XS_F * XS_NS + (i % (XS_F * XS_NS))] = make_double2((double)v.re, (double)v.im);
    }
  }
  if (bad) atomicOr(P.status, 1);
  __syncthreads();
#if XS_SPEC
  if (!P.single_step) {
    xs_spectrum(P, cta);
    for (int n = 0; n < P.npoints; ++n) {
      const cx* row = P.aft + ((size_t)cta * (P.nt + P.npoints) + P.nt + n) * XS_SPROW;
      xs_observe(row, row + GF, RED, n, t, P, wsum, cta, nctas, K, T, 1);
    }
  }
#endif
}

extern "C" __global__ void __launch_bounds__(XS_THREADS) xs_resident(const XsPathArgs P) {
  if (!xs_layout_ok(P.status)) return;
#if XS_GFIELD
  // one slice per CTA of the grid; CTAs loop over the trajectory tiles
  const int nctas = P.ntraj / XS_G;
  for (int c = blockIdx.x; c < nctas; c += gridDim.x) xs_resident_run(P, c, nctas);
#else
  xs_resident_run(P, blockIdx.x, gridDim.x);
#endif
}

// ---- uneven batch -------------------------------------------------------------
// Many independent problems of one compiled variant (same lattice, fields,
// expressions and tile) differing in trajectories, steps, time step, seed and
// the runtime scalars.  The persistent kernel pulls units (item, group of G
// trajectories) from a longest-first queue with one atomic per unit; the last
// unit of an item to finish reduces the item's partial sums in a fixed order,
// so the result does not depend on the schedule.
struct XsBatchItem {
  int ntraj, steps, npoints, seq;
  u32 seed;
  int block0;
  int nunits;
  short nc, checks;      // check pass (1 fine, 2 coarse) and p.checks of the item
  double wscale, vscale, dtr, t0;
  const double2* prop;   // [XS_PROP_COMPS][XS_NS] exp(L dtr / ipsteps) of this item
  double2* part;         // [npoints][nunits][XS_OBS_STRIDE] partial sums
  double2* av;           // [npoints][XS_OBS_STRIDE] means over the item's trajectories
  const double* params;  // runtime scalars of this item
  int* done;             // units finished
  const double2* prop2;  // exp(2 L dtr / ipsteps) of this item
};

struct XsBatchArgs {
  const XsBatchItem* items;
  const int2* units;     // (item, unit within item), longest first
  int nunits;
  int pad;
  int* next;             // queue head (zeroed before the launch)
  int* status;
  const cx* tmat;
  int tmat_off[4];
  cx* gfield;            // XS_GFIELD slices, one per CTA of the grid
};

extern "C" __global__ void __launch_bounds__(XS_THREADS) xs_batch(const XsBatchArgs B) {
  if (!xs_layout_ok(B.status)) return;
  __shared__ int s_unit, s_last;
  for (;;) {
    if (threadIdx.x == 0) s_unit = atomicAdd(B.next, 1);
    __syncthreads();
    const int u = s_unit;
    __syncthreads();
    if (u >= B.nunits) break;
    const int2 un = B.units[u];
    const XsBatchItem& it = B.items[un.x];
    XsPathArgs P;
    P.ntraj = it.ntraj;
    P.ens1 = it.ntraj;
    P.block0 = it.block0;
    P.nc = it.nc;
    P.checks = it.checks;
    P.npoints = it.npoints;
    P.steps = it.steps;
    P.seq = it.seq;
    P.seed = it.seed;
    P.pad0 = 0;
    P.wscale = it.wscale;
    P.vscale = it.vscale;
    P.dtr = it.dtr;
    P.t0 = it.t0;
    P.prop = it.prop;
    P.tmat = B.tmat;
#pragma unroll
    for (int d = 0; d < 4; ++d) P.tmat_off[d] = B.tmat_off[d];
    P.a_in = nullptr;
    P.a_out = nullptr;
    P.obs = it.part;
    P.status = B.status;
    P.single_step = 0;
    P.pad1 = 0;
    P.w_in = nullptr;
    P.params = it.params;
    P.gfield = B.gfield;
    P.prop2 = it.prop2;
    P.bval = nullptr;
    P.bda = nullptr;
    P.bval_n = 0;
    P.aft = nullptr;
    P.twt = nullptr;
    P.nt = 0;
    P.fscn = 0;
    P.raw = nullptr;
    P.kfilt = nullptr;
    P.rfilt = nullptr;
    P.kwscale = 0;
    P.kvscale = 0;
    xs_resident_run(P, un.y, it.nunits);
    // publish this unit's partial sums, then count it (threadFenceReduction pattern)
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(it.done, 1) == it.nunits - 1;
    __syncthreads();
    if (s_last && XS_OBS_STRIDE > 0) {
      __threadfence();
      const double inv = 1.0 / (double)it.ntraj;
      for (int k = threadIdx.x; k < it.npoints * XS_OBS_STRIDE; k += blockDim.x) {
        const int n = k / XS_OBS_STRIDE, q = k % XS_OBS_STRIDE;
        double re = 0, im = 0, cre = 0, cim = 0;
        for (int c = 0; c < it.nunits; ++c) {
          const double2 v = __ldcg(it.part + ((size_t)n * it.nunits + c) * XS_OBS_STRIDE + q);
          xs_kadd(re, cre, v.x);
          xs_kadd(im, cim, v.y);
        }
        it.av[k] = make_double2((re + cre) * inv, (im + cim) * inv);
      }
    }
    __syncthreads();
  }
}

// Block means over trajectories (xdata.m:84): av[b][n][k] = sum over the CTAs
// of block b of obs partials, divided by ens1.  Fixed summation order.
extern "C" __global__ void xs_obs_reduce(const double2* __restrict__ partial, double2* __restrict__ av,
                                         int npoints, int nctas, int ctas_per_block, int stride, double inv_ens) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = blockIdx.y;
  const int b = blockIdx.z;
  if (k >= stride) return;
  double sr = 0, si = 0, cr = 0, ci = 0;
  for (int c = 0; c < ctas_per_block; ++c) {
    const double2 v = partial[((size_t)n * nctas + (size_t)b * ctas_per_block + c) * stride + k];
    xs_kadd(sr, cr, v.x);
    xs_kadd(si, ci, v.y);
  }
  av[((size_t)b * npoints + n) * stride + k] = make_double2((sr + cr) * inv_ens, (si + ci) * inv_ens);
}
