"""The CPU oracle of the control-variate network: its backward pass agrees with
central finite differences of its own FP64 forward pass (no BF16 rounding)."""
import numpy as np

from oracle import mlp_ref


def _params(n_in, H, rng):
    sizes = [H * n_in, H, H * H, H, H * H, H, H, 1]
    return np.concatenate([rng.standard_normal(s) * (0.5 / np.sqrt(max(1, s // H))) for s in sizes])


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    n_in, H, B = 6, 5, 7
    P = _params(n_in, H, rng)
    x = rng.standard_normal((B, n_in))
    t = rng.standard_normal(B)
    _, g = mlp_ref.loss_and_grad(x, t, P, n_in, H, round_bf16=False)
    eps = 1e-6
    for i in rng.choice(P.size, 25, replace=False):
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += eps
        Pm[i] -= eps
        lp, _ = mlp_ref.loss_and_grad(x, t, Pp, n_in, H, round_bf16=False)
        lm, _ = mlp_ref.loss_and_grad(x, t, Pm, n_in, H, round_bf16=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) < 1e-6 * (1 + abs(fd)), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159265], dtype=np.float32)
    r = mlp_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
