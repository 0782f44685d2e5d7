// Learned control variate network (no counterpart in the reference): an MLP
// in -> H -> H -> H -> 1 with GELU activations, BF16 operands and FP32
// accumulation on the tensor cores, trained with hand-written forward,
// backward, loss and Adam kernels.  Parameters are kept as an FP32 master
// vector.  The hidden layers' forward GEMMs run on the sm_100a tensor cores
// (tcgen05.mma, accumulator in tensor memory, operand tiles brought into
// shared memory by the Tensor Memory Accelerator) whenever in is a multiple
// of 64 and H a multiple of 16 up to 256: the weights are converted to BF16
// once per call and the activations travel between layers as BF16.  The
// backward GEMMs, and other shapes, use warp-level BF16 MMA (wmma) with the
// FP32 operands rounded to BF16 when a tile is staged in shared memory.
//
// Parameter vector: W1[H][in], b1[H], W2[H][H], b2[H], W3[H][H], b3[H], w4[H], b4.
// Workspace (FP32): per hidden layer l = 1..3: Z_l[B][H] (pre-activation),
// A_l[B][H] (GELU output); then y[B]; then two [B][H] gradient buffers.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <cstddef>
#include <mutex>

#include "xs_mlp.hpp"

using namespace nvcuda;

namespace {

constexpr int TM = 64, TN = 64, TK = 32;  // CTA tile; 4 warps, each 32x32 (2x2 wmma 16x16 tiles)
constexpr int LDA = TK + 8, LDB = TN + 8, LDC = TN + 4;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// C[M][N] = sum_k A(m,k) B(k,n) (+ bias[n]) with
//   A(m,k) = TA ? A[k*lda + m] : A[m*lda + k],  B(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n].
// EPI 0: C = acc (+bias);  EPI 1: Z = acc + bias, C2 = gelu(Z).
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(128) gemm_bf16(const float* __restrict__ A, const float* __restrict__ B,
                                                 const float* __restrict__ bias, float* __restrict__ C,
                                                 float* __restrict__ C2, int M, int N, int K, int lda, int ldb,
                                                 int ldc) {
  __shared__ __align__(32) __nv_bfloat16 As[TM * LDA];
  __shared__ __align__(32) __nv_bfloat16 Bs[TK * LDB];
  __shared__ __align__(32) float Cs[TM * LDC];
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  const int warp = threadIdx.x >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) wmma::fill_fragment(acc[i][j], 0.0f);
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int i = threadIdx.x; i < TM * TK; i += blockDim.x) {
      const int mm = TA ? i % TM : i / TK, kk = TA ? i / TM : i % TK;
      const int gm = m0 + mm, gk = k0 + kk;
      float v = 0.f;
      if (gm < M && gk < K) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
      As[mm * LDA + kk] = __float2bfloat16_rn(v);
    }
    for (int i = threadIdx.x; i < TK * TN; i += blockDim.x) {
      const int kk = TB ? i % TK : i / TN, nn = TB ? i / TK : i % TN;
      const int gk = k0 + kk, gn = n0 + nn;
      float v = 0.f;
      if (gk < K && gn < N) v = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
      Bs[kk * LDB + nn] = __float2bfloat16_rn(v);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; kk += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa[2];
      wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) wmma::load_matrix_sync(fa[i], As + (wm + 16 * i) * LDA + kk, LDA);
#pragma unroll
      for (int j = 0; j < 2; ++j) wmma::load_matrix_sync(fb[j], Bs + kk * LDB + wn + 16 * j, LDB);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) wmma::mma_sync(acc[i][j], fa[i], fb[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
      wmma::store_matrix_sync(Cs + (wm + 16 * i) * LDC + wn + 16 * j, acc[i][j], LDC, wmma::mem_row_major);
  __syncthreads();
  for (int i = threadIdx.x; i < TM * TN; i += blockDim.x) {
    const int mm = i / TN, nn = i % TN, gm = m0 + mm, gn = n0 + nn;
    if (gm >= M || gn >= N) continue;
    float v = Cs[mm * LDC + nn] + (bias ? bias[gn] : 0.f);
    C[(size_t)gm * ldc + gn] = v;
    if (EPI == 1) C2[(size_t)gm * ldc + gn] = gelu(v);
  }
}

// y[b] = sum_h A[b][h] w[h] + c   (one warp per row)
__global__ void head_forward(const float* __restrict__ A, const float* __restrict__ w, const float* __restrict__ c,
                             float* __restrict__ y, int B, int H) {
  const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= B) return;
  float s = 0.f;
  for (int h = lane; h < H; h += 32) s += __bfloat162float(__float2bfloat16_rn(A[(size_t)row * H + h])) *
                                         __bfloat162float(__float2bfloat16_rn(w[h]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s + c[0];
}

// MSE loss 1/B sum (y - t)^2: dy = 2 (y - t) / B, loss accumulated in FP64.
__global__ void mse_grad(const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy,
                         double* __restrict__ loss, int B) {
  double part = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x) {
    const float r = y[i] - t[i];
    dy[i] = 2.0f * r / (float)B;
    part += (double)r * r / B;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, part);
}

// head backward: dA[b][h] = dy[b] * w[h] * gelu'(Z[b][h]) (the next layer's dZ);
// dw[h] = sum_b dy[b] A[b][h]; dc = sum_b dy[b].  Column sums: one thread per h.
__global__ void head_backward_dz(const float* __restrict__ dy, const float* __restrict__ w,
                                 const float* __restrict__ Z, float* __restrict__ dZ, int B, int H) {
  const size_t n = (size_t)B * H;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / H), h = (int)(i % H);
    dZ[i] = dy[b] * __bfloat162float(__float2bfloat16_rn(w[h])) * gelu_d(Z[i]);
  }
}

__global__ void colsum(const float* __restrict__ X, const float* __restrict__ wrow, float* __restrict__ out, int B,
                       int H) {
  // out[h] = sum_b X[b][h] * (wrow ? wrow[b] : 1)   (FP64 accumulation, fixed order)
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= H) return;
  double s = 0;
  for (int b = 0; b < B; ++b) s += (double)X[(size_t)b * H + h] * (wrow ? (double)wrow[b] : 1.0);
  out[h] = (float)s;
}

__global__ void scalar_sum(const float* __restrict__ x, float* __restrict__ out, int n) {
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < (int)(blockDim.x + 31) / 32; ++i) t += red[i];
    out[0] = (float)t;
  }
}

// dZ = dA * gelu'(Z)
__global__ void gelu_backward(const float* __restrict__ dA, const float* __restrict__ Z, float* __restrict__ dZ,
                              size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dZ[i] = dA[i] * gelu_d(Z[i]);
}

// Adam (Kingma & Ba, 2015) with decoupled weight decay wd (Loshchilov & Hutter, 2019).
__global__ void adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                     size_t n, float lr, float b1, float b2, float eps, float c1, float c2, float wd) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i]);
  }
}

// ---- hidden layer on the tensor cores (tcgen05) ------------------------------------
// Z[b][n] = sum_k A[b][k] W[n][k] + bias[n] for one tile of 128 rows b and all N
// columns.  A (BF16 [B][K]) and W (BF16 [N][K]) are K-major; the Tensor Memory
// Accelerator copies 64-column slices of both (128-byte rows, 128-byte swizzle)
// into a two-stage shared-memory ring, one thread issues tcgen05.mma
// (M = 128, N, K = 16, BF16 x BF16 -> FP32) into an accumulator of N tensor-memory
// columns, and eight warps read it back (tcgen05.ld; a warp reaches the 32 lanes =
// rows of its sub-partition, two warps split the columns) for the epilogue: bias,
// GELU, BF16 activations for the next layer, and in
// training the FP32 pre-activation and activation for the backward pass.  Every
// wait on an mbarrier is bounded: on a timeout the CTA sets status bit 0, waits
// (bounded) for its copies and products in flight, frees its tensor memory and
// returns.
namespace tc {
constexpr int BM = 128, BK = 64, STAGES = 2;
constexpr int WAIT_LIMIT = 1 << 24;

struct __align__(64) Tmap {
  unsigned long long w[16];
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  for (int it = 0; it < WAIT_LIMIT; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load(const Tmap* tm, unsigned dst, unsigned bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"((unsigned long long)tm), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// shared-memory matrix descriptor: K-major rows of 128 bytes with the 128-byte swizzle,
// 8-row groups 1024 bytes apart (stride byte offset), descriptor version 1, base offset 0
__device__ __forceinline__ unsigned long long sdesc(unsigned addr) {
  return (unsigned long long)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

template <bool TRAIN>
__global__ void __launch_bounds__(256, 1)
    layer_tc(const __grid_constant__ Tmap tA, const __grid_constant__ Tmap tW, int B, int K, int N, int ncols,
             const float* __restrict__ bias, float* __restrict__ Z, float* __restrict__ Af,
             __nv_bfloat16* __restrict__ Ab, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char dsm[];
  unsigned char* base = (unsigned char*)(((size_t)dsm + 1023) & ~(size_t)1023);
  const unsigned a_bytes = BM * BK * 2, w_bytes = (unsigned)N * BK * 2, stage_bytes = a_bytes + w_bytes;
  unsigned long long* bars = (unsigned long long*)(base + STAGES * stage_bytes);  // full[2], empty[2], done
  unsigned* tslot = (unsigned*)(bars + 2 * STAGES + 1);
  float* sbias = (float*)(tslot + 4);  // N bias values
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < N; i += blockDim.x) sbias[i] = bias[i];
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2 * STAGES + 1; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bars + i)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tslot;
  const int m0 = blockIdx.x * BM, nk = K / BK;
  const unsigned full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES), done = smem_u32(bars + 2 * STAGES);
  const unsigned sbase = smem_u32(base);
  // instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N, M = 128
  const unsigned idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(BM >> 4) << 24);
  __shared__ int s_ok;
  bool ok = true;
  if (threadIdx.x == 0) {
    auto issue = [&](int kb) {
      const int s = kb % STAGES;
      const unsigned bar = full0 + 8u * s, dst = sbase + s * stage_bytes;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(stage_bytes) : "memory");
      tma_load(&tA, dst, bar, kb * BK, m0);
      tma_load(&tW, dst + a_bytes, bar, kb * BK, 0);
    };
    int issued = 0;
    for (; issued < nk && issued < STAGES; ++issued) issue(issued);
    for (int kb = 0; kb < nk && ok; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(full0 + 8u * s, (unsigned)((kb / STAGES) & 1))) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned a0 = sbase + s * stage_bytes, w0 = a0 + a_bytes;
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const unsigned long long da = sdesc(a0 + kk * 32), dw = sdesc(w0 + kk * 32);
        const unsigned acc = (kb > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(da), "l"(dw), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(empty0 + 8u * s)
                   : "memory");
      if (issued < nk) {  // refill this stage once its products have read it
        if (!mbar_wait(empty0 + 8u * s, (unsigned)((kb / STAGES) & 1))) {
          ok = false;
          break;
        }
        issue(issued++);
      }
    }
    // the done barrier completes when every product issued so far has finished
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done) : "memory");
    if (!ok) {
      atomicOr(status, 1);
      // copies still in flight complete on their full barriers: wait for them (bounded) before leaving
      for (int kb = 0; kb < issued; ++kb) mbar_wait(full0 + 8u * (kb % STAGES), (unsigned)((kb / STAGES) & 1));
    }
    s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  ok = s_ok != 0;
  const bool fin = mbar_wait(done, 0);
  if (!fin && lane == 0) atomicOr(status, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (__all_sync(0xffffffffu, fin) && ok) {
    // warps w and w + 4 share the 32 accumulator lanes (rows) of sub-partition w % 4 and
    // split the N columns in 16-column chunks
    const int sub = warp & 3, half = warp >> 2, nch = N / 16, ch0 = half ? (nch + 1) / 2 : 0,
              ch1 = half ? nch : (nch + 1) / 2;
    const int row = m0 + 32 * sub + lane;
    for (int ch = ch0; ch < ch1; ++ch) {
      const int c0 = 16 * ch;
      unsigned r[16];
      const unsigned taddr = tmem + ((unsigned)(32 * sub) << 16) + (unsigned)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < B) {
        __align__(16) float z[16], g[16];
        __align__(16) __nv_bfloat16 gb[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          z[j] = __uint_as_float(r[j]) + sbias[c0 + j];
          g[j] = gelu(z[j]);
          gb[j] = __float2bfloat16_rn(g[j]);
        }
        const size_t o = (size_t)row * N + c0;
        if (TRAIN) {
#pragma unroll
          for (int j = 0; j < 16; j += 4) {
            *(float4*)(Z + o + j) = *(const float4*)(z + j);
            *(float4*)(Af + o + j) = *(const float4*)(g + j);
          }
        }
        *(uint4*)(Ab + o) = *(const uint4*)gb;
        *(uint4*)(Ab + o + 8) = *(const uint4*)(gb + 8);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

__global__ void to_bf16(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// y[b] = sum_h A[b][h] w[h] + c over BF16 activations (one warp per row)
__global__ void head_forward_bf16(const __nv_bfloat16* __restrict__ A, const float* __restrict__ w,
                                  const float* __restrict__ c, float* __restrict__ y, int B, int H) {
  const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= B) return;
  float s = 0.f;
  for (int h = lane; h < H; h += 32)
    s += __bfloat162float(A[(size_t)row * H + h]) * __bfloat162float(__float2bfloat16_rn(w[h]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s + c[0];
}

typedef CUresult (*PFN_encode)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                               const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

PFN_encode encoder() {
  static PFN_encode fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_encode)p;
  });
  return fn;
}

// 2D BF16 tensor [rows][cols] (cols contiguous), box 64 columns x box_rows rows, 128-byte swizzle
bool make_map(Tmap* m, const void* ptr, int rows, int cols, int box_rows) {
  PFN_encode enc = encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc((CUtensorMap*)m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t smem_bytes(int N) { return 1024 + (size_t)STAGES * (BM * BK * 2 + (size_t)N * BK * 2) + 64 + 4 * (size_t)N; }

int* status_buf() {
  static int* p = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) p = nullptr;
  });
  return p;
}
}  // namespace tc

bool tc_shape_ok(int in, int H) { return in % tc::BK == 0 && H % 16 == 0 && H >= 16 && H <= 256; }

struct Layout {
  size_t W[4], b[4], nparams;
  size_t Z[3], A[3], y, g1, g2, nwork;
  size_t xb, ab[3], wb[3];  // BF16 copies (offsets in floats, 256-byte aligned): x, activations, weights
};

Layout layout(int in, int H, int B) {
  Layout L{};
  size_t o = 0;
  L.W[0] = o; o += (size_t)H * in; L.b[0] = o; o += H;
  L.W[1] = o; o += (size_t)H * H; L.b[1] = o; o += H;
  L.W[2] = o; o += (size_t)H * H; L.b[2] = o; o += H;
  L.W[3] = o; o += H; L.b[3] = o; o += 1;
  L.nparams = o;
  size_t w = 0;
  for (int l = 0; l < 3; ++l) {
    L.Z[l] = w; w += (size_t)B * H;
    L.A[l] = w; w += (size_t)B * H;
  }
  L.y = w; w += B;
  L.g1 = w; w += (size_t)B * H;
  L.g2 = w; w += (size_t)B * H;
  auto al = [](size_t v) { return (v + 63) / 64 * 64; };
  w = al(w);
  L.xb = w; w = al(w + ((size_t)B * in + 1) / 2);
  for (int l = 0; l < 3; ++l) {
    L.ab[l] = w;
    w = al(w + ((size_t)B * H + 1) / 2);
  }
  for (int l = 0; l < 3; ++l) {
    L.wb[l] = w;
    w = al(w + ((size_t)H * (l == 0 ? in : H) + 1) / 2);
  }
  L.nwork = w;
  return L;
}

unsigned grid1(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

}  // namespace

size_t xs_mlp_layout(int in, int hidden, int batch, size_t* nparams) {
  Layout L = layout(in, hidden, batch);
  if (nparams) *nparams = L.nparams;
  return L.nwork;
}

// Forward pass on the tensor cores (tc_shape_ok): BF16 copies of x and the weights, three
// tcgen05 layers, the head on the CUDA cores.  train: also the FP32 pre-activations and
// activations the backward pass reads.
int forward_tc(int B, int in, int H, const float* x, const float* P, float* work, float* y, bool train,
               cudaStream_t st) {
  Layout L = layout(in, H, B);
  int* status = tc::status_buf();
  if (!status) return (int)cudaErrorMemoryAllocation;
  __nv_bfloat16* xb = (__nv_bfloat16*)(work + L.xb);
  tc::to_bf16<<<grid1((size_t)B * in), 256, 0, st>>>(x, xb, (size_t)B * in);
  for (int l = 0; l < 3; ++l) {
    const size_t n = (size_t)H * (l == 0 ? in : H);
    tc::to_bf16<<<grid1(n), 256, 0, st>>>(P + L.W[l], (__nv_bfloat16*)(work + L.wb[l]), n);
  }
  int ncols = 32;
  while (ncols < H) ncols <<= 1;
  const size_t smem = tc::smem_bytes(H);
  static std::once_flag attr;
  std::call_once(attr, [] {
    const int mx = (int)tc::smem_bytes(256);
    cudaFuncSetAttribute(tc::layer_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(tc::layer_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  });
  const __nv_bfloat16* a = xb;
  int K = in;
  const unsigned grid = (unsigned)((B + tc::BM - 1) / tc::BM);
  for (int l = 0; l < 3; ++l) {
    tc::Tmap tA, tW;
    const __nv_bfloat16* wb = (const __nv_bfloat16*)(work + L.wb[l]);
    if (!tc::make_map(&tA, a, B, K, tc::BM) || !tc::make_map(&tW, wb, H, K, H)) return (int)cudaErrorInvalidValue;
    __nv_bfloat16* ab = (__nv_bfloat16*)(work + L.ab[l]);
    if (train)
      tc::layer_tc<true><<<grid, 256, smem, st>>>(tA, tW, B, K, H, ncols, P + L.b[l], work + L.Z[l], work + L.A[l],
                                                  ab, status);
    else
      tc::layer_tc<false><<<grid, 256, smem, st>>>(tA, tW, B, K, H, ncols, P + L.b[l], nullptr, nullptr, ab, status);
    a = ab;
    K = H;
  }
  float* out = y ? y : work + L.y;
  tc::head_forward_bf16<<<(B + 7) / 8, 256, 0, st>>>(a, P + L.W[3], P + L.b[3], out, B, H);
  if (out != work + L.y) cudaMemcpyAsync(work + L.y, out, (size_t)B * 4, cudaMemcpyDeviceToDevice, st);
  return (int)cudaGetLastError();
}

int xs_mlp_forward_impl(int B, int in, int H, const float* x, const float* P, float* work, float* y,
                        cudaStream_t st, bool train) {
  if (tc_shape_ok(in, H)) return forward_tc(B, in, H, x, P, work, y, train, st);
  Layout L = layout(in, H, B);
  dim3 blk(128);
  dim3 g((H + TN - 1) / TN, (B + TM - 1) / TM);
  const float* a = x;
  int K = in;
  for (int l = 0; l < 3; ++l) {
    gemm_bf16<false, true, 1><<<g, blk, 0, st>>>(a, P + L.W[l], P + L.b[l], work + L.Z[l], work + L.A[l], B, H, K,
                                                  K, K, H);
    a = work + L.A[l];
    K = H;
  }
  float* out = y ? y : work + L.y;
  head_forward<<<(B + 7) / 8, 256, 0, st>>>(work + L.A[2], P + L.W[3], P + L.b[3], out, B, H);
  if (out != work + L.y) cudaMemcpyAsync(work + L.y, out, (size_t)B * 4, cudaMemcpyDeviceToDevice, st);
  return (int)cudaGetLastError();
}

int xs_mlp_backward_impl(int B, int in, int H, const float* x, const float* P, float* work, const float* target,
                         float* grad, double* loss, cudaStream_t st) {
  Layout L = layout(in, H, B);
  float* dy = work + L.g1;  // first B floats of g1 hold dy until layer 3's dZ is formed
  float* dZ = work + L.g2;
  cudaMemsetAsync(loss, 0, sizeof(double), st);
  mse_grad<<<grid1(B), 256, 0, st>>>(work + L.y, target, dy, loss, B);
  // head: dw4 = A3^T dy, db4 = sum dy, dZ3 = dy w4 gelu'(Z3)
  colsum<<<(H + 127) / 128, 128, 0, st>>>(work + L.A[2], dy, grad + L.W[3], B, H);
  scalar_sum<<<1, 256, 0, st>>>(dy, grad + L.b[3], B);
  head_backward_dz<<<grid1((size_t)B * H), 256, 0, st>>>(dy, P + L.W[3], work + L.Z[2], dZ, B, H);
  // dZ now holds the gradient of layer 3's pre-activation; dy is no longer needed, g1 is free.
  for (int l = 2; l >= 0; --l) {
    const float* aprev = l == 0 ? x : work + L.A[l - 1];
    const int K = l == 0 ? in : H;
    dim3 blk(128);
    // dW_l[h][k] = sum_b dZ[b][h] aprev[b][k]
    dim3 gw((K + TN - 1) / TN, (H + TM - 1) / TM);
    gemm_bf16<true, false, 0><<<gw, blk, 0, st>>>(dZ, aprev, nullptr, grad + L.W[l], nullptr, H, K, B, H, K, K);
    colsum<<<(H + 127) / 128, 128, 0, st>>>(dZ, nullptr, grad + L.b[l], B, H);
    if (l > 0) {
      // dA_{l-1}[b][k] = sum_h dZ[b][h] W_l[h][k]; then dZ_{l-1} = dA * gelu'(Z_{l-1})
      float* dAp = work + L.g1;
      dim3 gx((K + TN - 1) / TN, (B + TM - 1) / TM);
      gemm_bf16<false, false, 0><<<gx, blk, 0, st>>>(dZ, P + L.W[l], nullptr, dAp, nullptr, B, K, H, H, K, K);
      gelu_backward<<<grid1((size_t)B * K), 256, 0, st>>>(dAp, work + L.Z[l - 1], dZ, (size_t)B * K);
    }
  }
  return (int)cudaGetLastError();
}

int xs_mlp_adam_impl(size_t n, float* P, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                     int step, float wd, cudaStream_t st) {
  float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  adam<<<grid1(n), 256, 0, st>>>(P, g, m, v, n, lr, b1, b2, eps, c1, c2, wd);
  return (int)cudaGetLastError();
}

// Status of the tensor-core layers since the last call (bit 0: a bounded wait gave up),
// read synchronously on `st`, then cleared.
int xs_mlp_status(cudaStream_t st) {
  int* status = tc::status_buf();
  if (!status) return 0;
  int h = 0;
  if (cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return 0;
  if (cudaStreamSynchronize(st) != cudaSuccess) return 0;
  if (h) cudaMemsetAsync(status, 0, sizeof(int), st);
  return h;
}

int xs_mlp_uses_tensor_memory(int in, int hidden) { return tc_shape_ok(in, hidden) ? 1 : 0; }
