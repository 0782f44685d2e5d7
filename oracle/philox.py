"""Philox4x32-10 counter-based generator and the xSPDE noise mapping (NumPy).

TEST INFRASTRUCTURE ONLY: this is part of the CPU oracle that checks the CUDA
path.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it; the product never does.

Philox4x32-10 follows the published algorithm of Salmon, Moraes, Dror and Shaw,
"Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of
  (hi0, lo0) = mulhilo(M0, c0); (hi1, lo1) = mulhilo(M1, c2)
  c' = (hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0)
with the key bumped by the Weyl constants (W0, W1) between rounds.

The mapping of xSPDE noise draws onto Philox counters is this project's own
(the reference draws from MATLAB's ``rng(seed,'Threefry')`` stream,
Simulator/xensemble.m:26-31, which cannot be reproduced without MATLAB):

  key     = (seed mod 2^32, global ensemble block index b)
  counter = (site s, trajectory e in block, draw q, (component // 4) | seq << 16)

where ``s`` is the column-major (x fastest) lattice index, draw ``q = 0`` holds
the initial randoms of ``p.randomgen`` (Simulator/xrandom.m:20-23) and
``q >= 1`` the q-th call of ``p.noisegen`` in a path (Simulator/xnoise.m:29-38).
Each call gives four 32-bit words; words (0,1) and (2,3) each feed one
Box-Muller pair (Box and Muller, 1958) with uniforms u = (x + 1/2) 2^-32:
  z_even = sqrt(-2 ln u0) cos(2 pi u1),  z_odd = sqrt(-2 ln u0) sin(2 pi u1).
Component c of the call uses pair (c % 4) // 2 and the cos (even c) or sin
(odd c) branch.

k-space noises and randoms (knoises, krandoms: Simulator/xnoise.m:39-50,
xrandom.m:24-29) come from their own stream: the fourth counter word carries
bit 15 as well, (component // 4) | 0x8000 | seq << 16, with no site pairing;
the site index is the column-major index of the k-space lattice in FFT order.

Site pairing: when there are at most two components and the first space
dimension has an even number of points N1, one call serves two sites that
are N1/2 apart along x.  Site s with x index i1 uses the call whose site
counter is p = (i1 mod N1/2) + (N1/2) (s div N1), words (0,1) when
i1 < N1/2 and words (2,3) otherwise.  Otherwise each site has its own
calls, counter s, components in groups of four.
"""
import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint64(0x9E3779B9)
W1 = np.uint64(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)
SH = np.uint64(32)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10.  Inputs broadcast; returns four uint32 arrays."""
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) & MASK for x in (c0, c1, c2, c3))
    c0, c1, c2, c3 = np.broadcast_arrays(c0, c1, c2, c3)
    k0 = np.uint64(int(k0) & 0xFFFFFFFF)
    k1 = np.uint64(int(k1) & 0xFFFFFFFF)
    for r in range(10):
        if r:
            k0 = (k0 + W0) & MASK
            k1 = (k1 + W1) & MASK
        p0 = c0 * M0
        p1 = c2 * M1
        hi0, lo0 = p0 >> SH, p0 & MASK
        hi1, lo1 = p1 >> SH, p1 & MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0), lo1, (hi0 ^ c3 ^ k1), lo0
    return tuple(x.astype(np.uint32) for x in (c0, c1, c2, c3))


TWO_M32 = 2.0 ** -32


def uniform01(x):
    """(x + 1/2) 2^-32 in FP64: strictly inside (0, 1), exact in double."""
    return (x.astype(np.float64) + 0.5) * TWO_M32


def _boxmuller(w0, w1):
    u0 = uniform01(w0)
    u1 = uniform01(w1)
    r = np.sqrt(-2.0 * np.log(u0))
    th = 2.0 * np.pi * u1
    return r * np.cos(th), r * np.sin(th)


def normals(ncomp, nspace, nens, draw, block, seed, seq=0, n1=1, kstream=False):
    """Standard normals z[c, s, e] for one draw, shape (ncomp, nspace, nens).
    n1 is the number of points along the first space dimension (1 for SDEs);
    kstream selects the k-space stream."""
    out = np.empty((ncomp, nspace, nens), dtype=np.float64)
    e = np.arange(nens, dtype=np.uint64)[None, :]
    kbit = 0x8000 if kstream else 0
    if not kstream and ncomp <= 2 and n1 > 1 and n1 % 2 == 0 and nspace % n1 == 0:
        h = n1 // 2
        s = np.arange(nspace)
        i1 = s % n1
        pidx = (i1 % h + h * (s // n1)).astype(np.uint64)[:, None]
        hi = (i1 >= h)[:, None]
        w = philox4x32_10(pidx, e, draw, seq << 16, seed, block)
        za, zb = _boxmuller(np.where(hi, w[2], w[0]), np.where(hi, w[3], w[1]))
        out[0] = za
        if ncomp > 1:
            out[1] = zb
        return out
    s = np.arange(nspace, dtype=np.uint64)[:, None]
    for g in range((ncomp + 3) // 4):
        w = philox4x32_10(s, e, draw, g | kbit | (seq << 16), seed, block)
        for pair in range(2):
            c_even = 4 * g + 2 * pair
            if c_even >= ncomp:
                break
            u0 = uniform01(w[2 * pair])
            u1 = uniform01(w[2 * pair + 1])
            r = np.sqrt(-2.0 * np.log(u0))
            th = 2.0 * np.pi * u1
            out[c_even] = r * np.cos(th)
            if c_even + 1 < ncomp:
                out[c_even + 1] = r * np.sin(th)
    return out
