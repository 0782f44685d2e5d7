// Learned control variate network (no counterpart in the reference): an MLP
// in -> H -> H -> H -> 1 with GELU activations, BF16 operands and FP32
// accumulation on the tensor cores, trained with hand-written forward,
// backward, loss and Adam kernels.  Parameters are kept as an FP32 master
// vector and rounded to BF16 when a GEMM tile is staged in shared memory.
//
// Parameter vector: W1[H][in], b1[H], W2[H][H], b2[H], W3[H][H], b3[H], w4[H], b4.
// Workspace (FP32): per hidden layer l = 1..3: Z_l[B][H] (pre-activation),
// A_l[B][H] (GELU output); then y[B]; then two [B][H] gradient buffers.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <cstddef>

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

struct Layout {
  size_t W[4], b[4], nparams;
  size_t Z[3], A[3], y, g1, g2, nwork;
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

int xs_mlp_forward_impl(int B, int in, int H, const float* x, const float* P, float* work, float* y,
                        cudaStream_t st) {
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
