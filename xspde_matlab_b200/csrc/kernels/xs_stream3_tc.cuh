// Plane pass of the 3D streaming path on the tensor cores (sm_100a tcgen05), for
// 64 x 64 planes of one FP32 field component: the four dense DST/DCT transforms of
// an MP step (Applications/SPDE/xprop.m:18-42 with the reference's transforms
// xdct1.m ... xdst3.m, here the real matrices of xs_stream3.cuh) are GEMMs
//   D[r][k] = sum_n A[r][n] B[k][n],  r = part * 64 + line (part 0: real, 1: imaginary),
// A the plane's lines (128 rows of 64 values), B = M^T the transform (64 x 64),
// M = 128, N = 64, K = 64, issued by one thread as tcgen05.mma kind::tf32 into a
// 64-column tensor-memory accumulator.  FP32 accuracy from TF32 operands by the
// three-term split x = hi + lo (hi, lo TF32; Markidis et al., IPDPSW 2018):
// A B ~ A_lo B_hi + A_hi B_lo + A_hi B_hi, the small terms first.
//
// One plane, K state [ky][kx] in HBM -> K state:
//   T_x^-1 (lines: ky rows)  -> accumulator rows (part, ky), columns x
//   T_y^-1 (lines: x, the accumulator read back and written transposed) -> (part, x), y
//   MP step on the plane P[y][x] (xs3_mp_sites: noise, midpoint iterations,
//   Dirichlet mask), in the shared memory of the A tiles
//   T_x    (lines: y rows) -> (part, y), kx;  T_y (lines: kx) -> (part, kx), ky
//   -> P[ky][kx] -> HBM.
// Reading the accumulator (tcgen05.ld, a warp reaches the 32 lanes of its
// sub-partition) and writing the next A tile transposed is what moves the
// transform axis; each 32-lane warp writes one 128-byte operand row, so the
// stores are free of bank conflicts.
//
// Operand tiles are K-major with the 128-byte swizzle: K-block b (32 values =
// 128 bytes per row) of a tile of R rows at b * R * 128 bytes; row r at
// (r / 8) * 1024 + (r % 8) * 128; its 16-byte chunk c at chunk c ^ (r % 8).
// Shared memory (1024-byte aligned): B hi/lo of the four matrices (x inverse,
// y inverse, x forward, y forward; 16 KB each), A hi and A lo (32 KB each; A hi
// also holds the plane P between transforms), one mbarrier, the tensor-memory
// address.  One CTA of 512 threads per SM (persistent over planes); the next plane's K state
// is loaded into registers while the current one is transformed.  Every wait
// is bounded: on a timeout the CTA sets status bit 8, waits (bounded) for its
// products in flight, frees its tensor memory and returns.
#pragma once

#if XS3_TC
namespace tc3 {
constexpr int N = 64;                  // points per transformed dimension
constexpr unsigned BTILE = 64 * 256;   // bytes of a B tile (64 rows x 64 TF32)
constexpr unsigned ATILE = 128 * 256;  // bytes of an A tile (128 rows x 64 TF32)
constexpr unsigned OFF_A_HI = 8 * BTILE, OFF_A_LO = OFF_A_HI + ATILE, OFF_BAR = OFF_A_LO + ATILE;
constexpr unsigned SMEM_BYTES = OFF_BAR + 16 + 1024;  // + alignment slack
constexpr int WAIT_LIMIT = 1 << 24;
constexpr int TC3_NT = 512;                              // threads: 16 warps, four per accumulator sub-partition
constexpr int PER = 64 * 64 / TC3_NT;                    // plane elements per thread

__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) in a K-major 128-byte-swizzled tile of R rows
template <int R>
__device__ __forceinline__ unsigned sw_off(int r, int k) {
  return (unsigned)((k >> 5) * (R * 128) + (r >> 3) * 1024 + (r & 7) * 128 + ((((k & 31) >> 2) ^ (r & 7)) << 4) +
                    ((k & 3) << 2));
}

// x = hi + lo with hi and lo rounded to TF32 (as 32-bit patterns)
__device__ __forceinline__ void split_tf32(float x, u32& hi, u32& lo) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
  const float r = x - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

// value x at (r, k) of the hi and lo tiles
template <int R>
__device__ __forceinline__ void put(unsigned char* hi, unsigned char* lo, int r, int k, float x) {
  u32 h, l;
  split_tf32(x, h, l);
  const unsigned o = sw_off<R>(r, k);
  *(u32*)(hi + o) = h;
  *(u32*)(lo + o) = l;
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes
// apart, descriptor version 1
__device__ __forceinline__ unsigned long long sdesc(u32 addr) {
  return (unsigned long long)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// FP32 accumulator, TF32 A and B, both K-major, N = 64, M = 128
constexpr u32 IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((u32)(64 >> 3) << 17) | ((u32)(128 >> 4) << 24);

__device__ __forceinline__ void mma(u32 tmem, unsigned long long da, unsigned long long db, u32 acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(IDESC), "r"(acc)
      : "memory");
}

__device__ __forceinline__ bool mbar_wait(u32 bar, u32 parity) {
  for (int it = 0; it < WAIT_LIMIT; ++it) {
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

// D = A B^T for one transform in three TF32 products (one thread), then a commit that
// arrives on `bar` when they have finished.
__device__ __forceinline__ void gemm3(u32 tmem, u32 a_hi, u32 a_lo, u32 b_hi, u32 b_lo, u32 bar) {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
  for (int prod = 0; prod < 3; ++prod) {
    const u32 a = prod == 0 ? a_lo : a_hi, b = prod == 1 ? b_lo : b_hi;
#pragma unroll
    for (int kk = 0; kk < N / 8; ++kk) {  // K = 8 per product: 32 bytes of a 128-byte row
      const u32 ka = (u32)(kk >> 2) * ATILE / 2 + (u32)(kk & 3) * 32, kb = (u32)(kk >> 2) * BTILE / 2 + (u32)(kk & 3) * 32;
      mma(tmem, sdesc(a + ka), sdesc(b + kb), (prod | kk) ? 1u : 0u);
    }
  }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 16 accumulator columns c0 .. c0 + 15 of the lane this thread reaches
__device__ __forceinline__ void ld16(u32 taddr, float (&v)[16]) {
  u32 r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// x at byte p of the A hi tile and its TF32 remainder at the same place of the A lo tile
__device__ __forceinline__ void st2(unsigned char* p, float x) {
  u32 h, l;
  split_tf32(x, h, l);
  *(u32*)p = h;
  *(u32*)(p + ATILE) = l;
}

// Shared-memory writes of this thread visible to the tensor cores, then a CTA barrier.
__device__ __forceinline__ void publish() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
}
}  // namespace tc3

// One MP step (K state in, K state out) of every plane, the transforms on the tensor cores.
// mtc: the four transforms as FP32 matrices B_m[k][n] = M[n][k] (input n, output k),
// m = 0 x inverse, 1 y inverse, 2 x forward, 3 y forward.
extern "C" __global__ void __launch_bounds__(tc3::TC3_NT, 1) xs_p_nl_tc(const XsStreamArgs A, const float* __restrict__ mtc) {
  using namespace tc3;
  if (blockDim.x != TC3_NT || XS3_N1 != N || XS3_N2 != N) {
    if (threadIdx.x == 0) atomicOr(A.status, 2);
    return;
  }
  if (!xs_smem_ok(SMEM_BYTES, A.status)) return;
  unsigned char* base = (unsigned char*)(((size_t)xs_dsmem + 1023) & ~(size_t)1023);
  unsigned char *ahi = base + OFF_A_HI, *alo = base + OFF_A_LO;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int m = 0; m < 4; ++m)
    for (int i = tid; i < N * N; i += TC3_NT)
      put<64>(base + (2 * m) * BTILE, base + (2 * m + 1) * BTILE, i / N, i % N, mtc[m * N * N + i]);
  const u32 sb = smem_u32(base), bar = sb + OFF_BAR;
  u32* tslot = (u32*)(base + OFF_BAR + 8);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(64)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  publish();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const u32 tmem = *tslot;
  // this thread reaches accumulator row 32 * sub + lane = part * 64 + line, columns 16 * quarter ..
  const int sub = warp & 3, quarter = warp >> 2, part = sub >> 1, line = 32 * (sub & 1) + lane;
  const u32 taddr = tmem + ((u32)(32 * sub) << 16) + (u32)(16 * quarter);
  u32 phase = 0;
  bool ok = true;
  // D = A B_m^T with A published; false when the products did not finish in time
  auto round = [&](int m) -> bool {
    if (tid == 0) gemm3(tmem, sb + OFF_A_HI, sb + OFF_A_LO, sb + 2 * m * BTILE, sb + (2 * m + 1) * BTILE, bar);
    const bool done = mbar_wait(bar, phase);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (__syncthreads_or(!done)) return false;
    phase ^= 1u;
    return true;
  };
  // accumulator (part, line) x columns -> A rows (part, column), K = line.  Row
  // part * 64 + 16 quarter + j of column `line` lies at tp[j % 8] + 1024 (j / 8): the
  // rows' 8-row group advances by 1024 bytes, their position in it sets the swizzle
  unsigned char* tp[8];
#pragma unroll
  for (int jc = 0; jc < 8; ++jc) tp[jc] = ahi + sw_off<128>(part * N + 16 * quarter + jc, line);
  auto transpose_into_a = [&]() {
    float v[16];
    ld16(taddr, v);
#pragma unroll
    for (int j = 0; j < 16; ++j) st2(tp[j & 7] + 1024 * (j >> 3), v[j]);
    publish();
  };
  // accumulator (part, line) x columns -> plane P[column][line] (complex, in the A hi tile)
  auto into_plane = [&](float* P) {
    float v[16];
    ld16(taddr, v);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // every thread is past its reads of the A tiles' last products
#pragma unroll
    for (int j = 0; j < 16; ++j) P[2 * ((16 * quarter + j) * N + line) + part] = v[j];
    __syncthreads();
  };
  const size_t nplanes = (size_t)A.ntraj * XS3_N3;
  float2 cur[PER], nxt[PER];
  // the loads stay where they are written (volatile), so the next plane is in flight while
  // the current one is transformed
  auto load = [&](size_t pl, float2 (&r)[PER]) {
    const float2* g = reinterpret_cast<const float2*>(A.field + pl * XS3_NP);
#pragma unroll
    for (int jj = 0; jj < PER; ++jj)
      asm volatile("ld.global.cs.v2.f32 {%0, %1}, [%2];" : "=f"(r[jj].x), "=f"(r[jj].y) : "l"(g + tid + TC3_NT * jj));
  };
  // plane rows (part, row), K = column from PER complex values per thread: element
  // tid + 512 jj is row tid / 64 + 8 jj (its 8-row group jj, 1024 bytes apart; the
  // imaginary rows 64 further, 8192 bytes), column tid % 64
  static_assert(TC3_NT == 512 && N == 64, "row layout of rows_into_a");
  unsigned char* const rp = ahi + sw_off<128>(tid / N, tid % N);
  auto rows_into_a = [&](const float2 (&r)[PER]) {
#pragma unroll
    for (int jj = 0; jj < PER; ++jj) {
      st2(rp + 1024 * jj, r[jj].x);
      st2(rp + 1024 * jj + 8192, r[jj].y);
    }
    publish();
  };
  if ((size_t)blockIdx.x < nplanes) load(blockIdx.x, cur);
  for (size_t pl = blockIdx.x; pl < nplanes; pl += gridDim.x) {
    const int e = (int)(pl / XS3_N3), z = (int)(pl % XS3_N3);
    if (pl + gridDim.x < nplanes) load(pl + gridDim.x, nxt);
    rows_into_a(cur);  // K state [ky][kx]: rows (part, ky), K = kx
    if (!(ok = round(0))) break;  // T_x^-1 -> (part, ky) x x
    transpose_into_a();           // rows (part, x), K = ky
    if (!(ok = round(1))) break;  // T_y^-1 -> (part, x) x y
    float* P = reinterpret_cast<float*>(ahi);
    into_plane(P);  // P[y][x]
    xs3_mp_sites<N, TC3_NT>(A, reinterpret_cast<cx*>(P), e, z, tid);
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < PER; ++jj) cur[jj] = reinterpret_cast<const float2*>(P)[tid + TC3_NT * jj];
    __syncthreads();
    rows_into_a(cur);             // rows (part, y), K = x
    if (!(ok = round(2))) break;  // T_x -> (part, y) x kx
    transpose_into_a();           // rows (part, kx), K = y
    if (!(ok = round(3))) break;  // T_y -> (part, kx) x ky
    into_plane(P);                // P[ky][kx]
    float2* g = reinterpret_cast<float2*>(A.field + pl * XS3_NP);
#pragma unroll
    for (int jj = 0; jj < PER; ++jj) g[tid + TC3_NT * jj] = reinterpret_cast<const float2*>(P)[tid + TC3_NT * jj];
    __syncthreads();  // P read before the next plane's A tiles are written
#pragma unroll
    for (int jj = 0; jj < PER; ++jj) cur[jj] = nxt[jj];
  }
  if (!ok) {
    if (tid == 0) atomicOr(A.status, 8);
    mbar_wait(bar, phase);  // the products in flight (bounded)
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
  }
}
#endif  // XS3_TC
