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
