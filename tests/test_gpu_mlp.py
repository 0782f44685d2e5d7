"""Control-variate network kernels on the GPU against the CPU oracle
(oracle/mlp_ref.py): forward output and the loss gradient with respect to
every parameter (BF16 operands on both sides; tolerance 2e-3 relative, the
remaining difference being FP32 vs FP64 accumulation), and a fit on a problem
with a known smooth dependence showing the variance the network removes.
Shapes with n_in a multiple of 64 and H a multiple of 16 (up to 256) run the
hidden layers on the tcgen05 tensor cores -- (256, 256, 256) and
(128, 192, 1000), whose last 128-row tile is partly outside the batch --
the others on warp-level MMA."""
import ctypes

import numpy as np
import pytest

from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("n_in,H,B", [(256, 256, 256), (128, 192, 1000), (40, 72, 100)])
def test_forward_and_gradient_match_oracle(n_in, H, B):
    import torch
    from xspde_matlab_b200 import _lib
    from xspde_matlab_b200.cv import ControlVariateNet
    torch.manual_seed(0)
    net = ControlVariateNet(n_in, H, seed=1)
    net.params.add_(torch.randn_like(net.params) * 0.01)  # non-zero biases
    x = torch.randn(B, n_in, device="cuda")
    t = torch.randn(B, device="cuda")
    L = _lib.lib()
    work = torch.empty(L.xs_mlp_sizes(n_in, H, B, None), dtype=torch.float32, device="cuda")
    y = torch.empty(B, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.xs_mlp_forward(B, n_in, H, _ptr(x), _ptr(net.params), _ptr(work), _ptr(y), st))
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    grad = torch.zeros_like(net.params)
    _lib.check(L.xs_mlp_train_grad(B, n_in, H, _ptr(x), _ptr(net.params), _ptr(work), _ptr(t), _ptr(grad),
                                   _ptr(loss), st))
    torch.cuda.synchronize()
    P = net.params.cpu().numpy()
    y_ref, _, _ = mlp_ref.forward(x.cpu().numpy(), P, n_in, H)
    l_ref, g_ref = mlp_ref.loss_and_grad(x.cpu().numpy(), t.cpu().numpy(), P, n_in, H)
    assert np.max(np.abs(y.cpu().numpy() - y_ref)) < 2e-3 * np.max(np.abs(y_ref))
    assert abs(loss.item() - l_ref) < 2e-3 * l_ref
    g = grad.cpu().numpy()
    sizes = [H * n_in, H, H * H, H, H * H, H, H, 1]
    o = 0
    for s in sizes:
        ga, gb = g[o:o + s], g_ref[o:o + s]
        assert np.linalg.norm(ga - gb) <= 2e-3 * np.linalg.norm(gb) + 1e-9, (o, s)
        o += s


def test_training_removes_variance():
    import torch
    from xspde_matlab_b200.cv import ControlVariateNet, two_level
    torch.manual_seed(0)
    n_in = 64
    w = torch.randn(n_in, device="cuda") / np.sqrt(n_in)

    def observable(x, noise):
        s = x @ w
        return 1.0 + 0.3 * s + 0.1 * torch.tanh(2 * s) ** 2 + 0.05 * noise

    X = torch.randn(16384, n_in, device="cuda")
    f = observable(X, torch.randn(16384, device="cuda"))
    net = ControlVariateNet(n_in, 128, seed=2)
    net.fit(X, f, epochs=20, batch=512, lr=2e-3)
    Xt = torch.randn(4096, n_in, device="cuda")
    ft = observable(Xt, torch.randn(4096, device="cuda")).double()
    gt = net.predict(Xt)
    var_plain = float(ft.var())
    var_cv = float((ft - gt).var())
    assert var_cv < 0.1 * var_plain, (var_cv, var_plain)
    fresh = net.predict(torch.randn(1 << 18, n_in, device="cuda"))
    est, err = two_level(ft.cpu().numpy(), gt.cpu().numpy(), fresh.cpu().numpy(), 16)
    exact = 1.0 + 0.1 * float(torch.mean(torch.tanh(2 * torch.randn(1 << 22, device="cuda")) ** 2))
    assert abs(est - exact) < 5 * err + 1e-3
