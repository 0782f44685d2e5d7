// Launch arguments and helpers shared by the streaming kernels of 2D lattices
// (xs_stream.cuh: row and column passes) and of 3D lattices (xs_stream3.cuh:
// plane and z-line passes).  Included after the problem header and the
// generated drift/observable functions.
#pragma once

struct XsStreamArgs {
  int ntraj;      // trajectories in this launch
  int ens1;       // trajectories per block
  int block0;     // global index of the first block
  int seq;        // sequence index (Philox counter)
  u32 seed;
  int draw0;      // Philox draw of this step
  int draw1;      // >= 0: coarse pass, average draws draw0 and draw1 (xnoise.m:33-35)
  int m;          // column / z-line pass: power of the half-step propagator (1 or 2)
  int n;          // observation index
  int npoints;
  double wscale;  // sqrt(nscale * noisefactor)
  double vscale;  // sqrt(noisefactor)
  double dtr;     // step of this pass
  double t;       // time at the start of this step (or of the observation)
  cx* field;                 // [ntraj][F][NS]
  const double2* prop1;      // [PC][NS] exp(L dtr/ipsteps), site order (x fastest)
  const double2* prop2;      // [PC][NS] exp(2 L dtr/ipsteps)
  const double2* a_in;       // [ntraj][F][NS] FP64 or null
  double2* a_out;            // [ntraj][F][NS] FP64 or null
  double2* av;               // [nblocks][npoints][XS_OBS_STRIDE]
  double2* redpart;          // [ntraj][XS_NRG][XS_NRED] integrand sums per row group (2D) or plane (3D)
  int* status;
  const double* params;      // runtime values of the named scalars p.<name>
  const cx* tw_x;            // 2D: [RX*RX] four-step twiddles of the rows, built in FP64 on the host
  const cx* tw_y;            // 2D: [RY*RY] four-step twiddles of the columns
  double2* opart;            // [gridDim.z][nblocks][XS_NOUT_SITE * NS] per-split sums of the site observables
  cx* field2;                // RK4: the second field (a1, then a3) [ntraj][F][NS], K state
  int ndraw0, ndraw1;        // RK4 row pass 3 fused with the next step's pass 1: that step's draws
  int fuse;                  // RK4 row pass 3: 1 = also do the next step's pass 1
  const real* mat;           // 3D: real transform matrices [6][N][N] (x, y, z; forward, inverse), M[n*N + k]
  int xspace;                // 3D: 1 = the field is held in x space (initial field, before its first transform)
};

extern __shared__ __align__(16) unsigned char xs_dsmem[];  // sizes set at launch

// True when this launch's dynamic shared memory holds `need` bytes; otherwise
// the CTA records status bit 1 and must return without touching shared memory.
__device__ __forceinline__ bool xs_smem_ok(size_t need, int* status) {
  u32 dyn;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
  if ((size_t)dyn >= need) return true;
  if (threadIdx.x == 0) atomicOr(status, 2);
  return false;
}

// Scalar observables from per-trajectory reductions (NRG partial sums per
// trajectory: row groups in 2D, planes in 3D): CTA per block, fixed summation
// order over the parts and the trajectories.
template <int NRG>
__device__ __forceinline__ void xs_scalar_body(const XsStreamArgs& A) {
#if XS_NOUT_SCALAR > 0
  __shared__ double part[8][2 * XS_NOUT_SCALAR];
  const int b = blockIdx.x;
  if ((size_t)(b + 1) * A.ens1 > (size_t)A.ntraj || blockDim.x > 256) {
    if (threadIdx.x == 0) atomicOr(A.status, 2);
    return;
  }
  double acc[2 * XS_NOUT_SCALAR], cmp[2 * XS_NOUT_SCALAR];  // compensated per-thread sums
#pragma unroll
  for (int k = 0; k < 2 * XS_NOUT_SCALAR; ++k) acc[k] = cmp[k] = 0;
  for (int el = threadIdx.x; el < A.ens1; el += blockDim.x) {
    const int e = b * A.ens1 + el;
    cx red[XS_NRED > 0 ? XS_NRED : 1];
#pragma unroll
    for (int k = 0; k < XS_NRED; ++k) {
      double re = 0, im = 0;
      for (int g = 0; g < NRG; ++g) {
        const double2 q = A.redpart[((size_t)e * NRG + g) * XS_NRED + k];
        re += q.x;
        im += q.y;
      }
      red[k] = mkcx((real)re, (real)im);
    }
    cx o[XS_NOUT_SCALAR];
    xs_obs_scalar(red, (real)A.t, A.params, o);
#pragma unroll
    for (int k = 0; k < XS_NOUT_SCALAR; ++k) {
      xs_kadd(acc[2 * k], cmp[2 * k], (double)o[k].re);
      xs_kadd(acc[2 * k + 1], cmp[2 * k + 1], (double)o[k].im);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 2 * XS_NOUT_SCALAR; ++k) {
    const double s = xs_warp_sum(acc[k] + cmp[k]);
    if (lane == 0) part[warp][k] = s;
  }
  __syncthreads();
  if (threadIdx.x < XS_NOUT_SCALAR) {
    double re = 0, im = 0;
    for (int q = 0; q < 8; ++q) {
      re += part[q][2 * threadIdx.x];
      im += part[q][2 * threadIdx.x + 1];
    }
    const double inv = 1.0 / (double)A.ens1;
    A.av[((size_t)b * A.npoints + A.n) * XS_OBS_STRIDE + (size_t)XS_NOUT_SITE * XS_NS + threadIdx.x] =
        make_double2(re * inv, im * inv);
  }
#endif
}

// Block means of the site observables from the nsplit partial sums of the
// observation pass (compensated, fixed order): grid (ceil(NOUT_SITE * NS / 256), nblocks).
extern "C" __global__ void __launch_bounds__(256) xs_x_obs_combine(const XsStreamArgs A, int nsplit) {
#if XS_NOUT_SITE > 0
  constexpr size_t M = (size_t)XS_NOUT_SITE * XS_NS;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (i >= M) return;
  double re = 0, im = 0, cre = 0, cim = 0;
  for (int z = 0; z < nsplit; ++z) {
    const double2 q = A.opart[((size_t)z * gridDim.y + b) * M + i];
    xs_kadd(re, cre, q.x);
    xs_kadd(im, cim, q.y);
  }
  const double inv = 1.0 / (double)A.ens1;
  A.av[((size_t)b * A.npoints + A.n) * XS_OBS_STRIDE + i] = make_double2((re + cre) * inv, (im + cim) * inv);
#endif
}
