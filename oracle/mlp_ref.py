"""CPU oracle of the learned control variate network (test infrastructure only).

TEST INFRASTRUCTURE ONLY: checks the device MLP kernels of xspde_matlab_b200.
Only tests/ and bench.py's CPU legs may import it.

FP64 NumPy forward and backward of the MLP in -> H -> H -> H -> 1 (GELU) with
the device's rounding points: every GEMM operand is rounded to BF16 (round to
nearest even), accumulation and epilogues in higher precision.  Parameter
vector order: W1[H][in], b1[H], W2[H][H], b2[H], W3[H][H], b3[H], w4[H], b4.
The network has no counterpart in the reference.
"""
import math

import numpy as np


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = x.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    u = ((u + rounding) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _erf(x):
    return np.vectorize(math.erf)(x)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def unpack(P, n_in, H):
    P = np.asarray(P, dtype=np.float64)
    o = 0
    out = []
    for rows, cols in ((H, n_in), (H, H), (H, H)):
        W = P[o:o + rows * cols].reshape(rows, cols)
        o += rows * cols
        b = P[o:o + rows]
        o += rows
        out.append((W, b))
    w4 = P[o:o + H]
    o += H
    b4 = P[o]
    return out, w4, b4


def forward(x, P, n_in, H, round_bf16=True):
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    layers, w4, b4 = unpack(P, n_in, H)
    a = np.asarray(x, dtype=np.float32)
    cache = []
    for W, b in layers:
        z = r(a) @ r(W).T + b
        z = z.astype(np.float32).astype(np.float64) if round_bf16 else z
        cache.append((a, z))
        a = gelu(z)
        a = a.astype(np.float32).astype(np.float64) if round_bf16 else a
    y = r(a) @ r(w4) + b4
    return y, cache, a


def loss_and_grad(x, t, P, n_in, H, round_bf16=True):
    """MSE loss and its gradient with respect to the parameter vector."""
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    layers, w4, b4 = unpack(P, n_in, H)
    y, cache, a3 = forward(x, P, n_in, H, round_bf16)
    B = y.shape[0]
    res = y - np.asarray(t, dtype=np.float64)
    loss = np.mean(res ** 2)
    dy = 2.0 * res / B
    g_w4 = a3.T @ dy
    g_b4 = dy.sum()
    dz = dy[:, None] * r(w4)[None, :] * gelu_d(cache[2][1])
    grads = [None] * 3
    for l in (2, 1, 0):
        a_prev, z = cache[l]
        W, b = layers[l]
        gW = r(dz).T @ r(a_prev)
        gb = dz.sum(axis=0)
        grads[l] = (gW, gb)
        if l > 0:
            da = r(dz) @ r(W)
            dz = da * gelu_d(cache[l - 1][1])
    flat = []
    for gW, gb in grads:
        flat += [gW.reshape(-1), gb]
    flat += [g_w4, np.array([g_b4])]
    return loss, np.concatenate(flat)
