"""What the learned control variate gains, on pairs the solver generates.

A Kubo oscillator, da = i a w dt (Examples/SDE_1D/Kubo2.m's equation; MP,
Stratonovich), observed as Re a(T) = cos(W_T): an even, nonlinear function of
the Wiener increments.  The network inputs are the device's own projections of
the increments that drove each trajectory (xs_noise_features: one feature per
step, 64 steps), so every (features, observable) pair comes from the solver.
A linear least-squares control variate removes almost nothing (cos is even, so
it is uncorrelated with every feature); the MLP trained by the project's
tcgen05 forward and backward kernels removes most of the variance.  The
two-level estimate mean_N(f - g) + mean_M(g) on the validation trajectories
agrees with the plain mean of the independent training trajectories (the
same discretisation; the continuum value exp(-T/2) differs from it by the
O(dt) bias of MP's midpoint phase), within five of xSPDE's block sampling
errors (Simulator/xsim.m:95), with a smaller error than the plain estimate
on the same trajectories.
"""
import ctypes
import math

import pytest

pytestmark = pytest.mark.gpu

T = 1.0
KUBO = dict(dimensions=1, points=[65], ranges=[T], steps=1, noises=1, method="MP", checks=0,
            deriv="@(a,w,p) 1i*a.*w", initial="@(w,p) 1+0*w", observe=["@(a,p) real(a)"])


def _pairs(first_block, n):
    """Observable at t = T and the 64 noise features of n single-trajectory blocks."""
    import torch
    from xspde_matlab_b200 import GpuPath, _lib, xpreferences
    L = _lib.lib()
    path = GpuPath(xpreferences([dict(KUBO, ensembles=[1, n, 1])])[0])
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    av = torch.zeros((n, path.per_block // 2, 2), dtype=torch.float64, device="cuda")
    _lib.check(L.xs_run_path_device(path.h, first_block, n, 1, None, ctypes.c_void_p(av.data_ptr()), None, st))
    X = torch.empty((n, 64), dtype=torch.float32, device="cuda")
    region = (ctypes.c_int * 6)(0, 0, 1, 1, 1, 1)
    # draw q feeds step q (xpath.m:34): steps 1..64 are the 64 integration steps
    _lib.check(L.xs_noise_features(path.h, first_block, n, region, 1, 1, 64, 0.0, ctypes.c_void_p(X.data_ptr()), st))
    _lib.check(L.xs_sync(path.h))
    return av[:, -1, 0].clone(), X


def test_mlp_control_variate_beats_linear_on_solver_pairs():
    import torch
    from xspde_matlab_b200.cv import ControlVariateNet, two_level
    ntrain, nval = 1 << 15, 1 << 13
    f_tr, X_tr = _pairs(0, ntrain)
    f_va, X_va = _pairs(ntrain, nval)
    # the features are what the solver integrated: their sum is W_T / sqrt(dt) up to scale
    assert abs(float(X_tr.mean())) < 0.02 and abs(float(X_tr.var()) - 1) < 0.02
    # linear least squares on the features
    A = torch.cat([X_tr.double(), torch.ones(ntrain, 1, dtype=torch.float64, device="cuda")], 1)
    coef = torch.linalg.solve(A.T @ A, A.T @ f_tr.unsqueeze(1))[:, 0]

    def g_lin(X):
        return X.double() @ coef[:-1] + coef[-1]
    var_plain = float(f_va.var())
    var_lin = float((f_va - g_lin(X_va)).var())
    net = ControlVariateNet(64, 64, seed=3)
    net.fit(X_tr, f_tr, epochs=12, batch=1024, lr=2e-3)
    g_va = net.predict(X_va)
    var_mlp = float((f_va - g_va).var())
    assert var_lin > 0.9 * var_plain, (var_lin, var_plain)  # the even dependence is invisible to a linear fit
    assert var_mlp < 0.25 * var_lin, (var_mlp, var_lin)     # the network removes most of the variance
    fresh = net.predict(torch.randn(1 << 20, 64, device="cuda"))
    est, err = two_level(f_va.cpu().numpy(), g_va.cpu().numpy(), fresh.cpu().numpy(), 16)
    ref = float(f_tr.mean())
    ref_err = math.sqrt(float(f_tr.var()) / ntrain)
    assert abs(est - ref) < 5 * math.sqrt(err ** 2 + ref_err ** 2), (est, err, ref, ref_err)
    assert abs(ref - math.exp(-T / 2)) < 0.02  # the continuum value, up to MP's O(dt) bias
    plain_err = math.sqrt(var_plain / nval)
    assert err < 0.6 * plain_err, (err, plain_err)
