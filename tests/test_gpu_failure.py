"""Failure detection without a GPU fault.

The reference's only failure mode on this path is numerical: a trajectory
that diverges turns into NaN/Inf and silently pollutes the ensemble means
(MATLAB arithmetic does not stop; Applications/SPDE/xtransform.m:51 is its one
explicit error).  The device path instead reports it: every kernel family
sets status bit 0 when a final field is non-finite, and the C ABI returns
XS_ERR_NAN from xs_run_path, or from xs_sync after xs_run_path_device.  The
divergence here is a finite-time blow-up of da/dt = a^3 from a = 10 (it
reaches infinity at t = 1/200): ordinary floating-point overflow, nothing
that faults.  The same device context keeps working afterwards.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

XS_ERR_NAN = -5


def _healthy_runs():
    from xspde_matlab_b200 import GpuPath, xpreferences
    p = xpreferences([dict(dimensions=1, points=[5], ranges=[1.0], steps=4, ensembles=[8, 1, 1], noises=1,
                           method="MP", deriv="@(a,w,p) -a + w", initial="@(w,p) 1+0*w",
                           observe=["@(a,p) real(a)"])])[0]
    av, _ = GpuPath(p).run_path(0, 1, 1)
    assert np.all(np.isfinite(av[0][0]))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_diverging_sde_returns_nan_status(precision):
    from xspde_matlab_b200 import GpuPath, _lib, xpreferences
    p = xpreferences([dict(dimensions=1, points=[5], ranges=[1.0], steps=4, ensembles=[16, 2, 1], noises=1,
                           method="MP", precision=precision, deriv="@(a,w,p) a.^3 + 0.01*w",
                           initial="@(w,p) 10+0*w", observe=["@(a,p) real(a)"])])[0]
    path = GpuPath(p)
    with pytest.raises(_lib.XsError) as ei:
        path.run_path(0, 2, 1)
    assert ei.value.code == XS_ERR_NAN
    _healthy_runs()


def test_diverging_streaming_lattice_returns_nan_from_sync():
    """64x64 lattice forced onto the streaming kernels; the launch itself
    returns XS_OK (it only enqueues work) and xs_sync reports XS_ERR_NAN,
    set by the observation pass."""
    import torch

    from xspde_matlab_b200 import GpuPath, _lib, xpreferences
    p = xpreferences([dict(dimensions=3, points=[3, 64, 64], ranges=[0.2, 10.0, 10.0], steps=2, ensembles=[4, 1, 1],
                           noises=2, method="MP", precision="fp32",
                           deriv="@(a,w,p) a.^3 + 0.01*w(1,:)", initial="@(v,p) 10 + 0*v(1,:)",
                           linear="@(p) 0.1i*(p.Dx.^2+p.Dy.^2)", observe=["@(a,p) abs(a).^2"])])[0]
    path = GpuPath(p, path_kind=2)
    L = _lib.lib()
    av = torch.zeros((path.per_block,), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    # no final field requested: the observation pass is what notices the divergence
    rc = L.xs_run_path_device(path.h, 0, 1, 1, None, ctypes.c_void_p(av.data_ptr()), None,
                              ctypes.c_void_p(st.cuda_stream))
    assert rc == 0
    assert L.xs_sync(path.h) == XS_ERR_NAN
    msg = ctypes.create_string_buffer(512)
    L.xs_last_error(msg, 512)
    assert b"non-finite" in msg.value
    _healthy_runs()
