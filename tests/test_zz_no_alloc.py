"""The allocation-free entry point, xs_run_path_device_noalloc.

Callers that may not call cudaMalloc -- a MATLAB MEX function that leaves
device memory to MATLAB's gpuArray allocator, code being recorded into a CUDA
graph, a service with a fixed memory budget -- run the resident path with its
observable partial sums in the library's fixed 16 MiB device array.  This
test checks, through the C ABI, that two calls in a row give the same block
means as the allocating entry point xs_run_path_device (FP64 tolerance of
the other GPU tests, 1e-10 relative), and that a launch whose partial sums
exceed the fixed array is refused with a clear error.  The file name makes
pytest collect it last.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

SMALL = dict(dimensions=2, points=[11, 64], ranges=[1.0, 10.0], steps=4, ensembles=[8, 2, 1], noises=2,
             method="MP", checks=1,
             deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2",
             observe=["@(a,p) a.*conj(a)", "@(a,p) Int(abs(a).^2, p)"])


def _path(p):
    from xspde_matlab_b200 import GpuPath, xpreferences
    return GpuPath(xpreferences([p])[0], path_kind=1)


def _av(path, nblocks):
    import torch
    P = path.p
    row = sum(ln * (P.nspace if sp else 1) for ln, sp, *_ in path.obs)
    return torch.zeros((nblocks, P.points[0], row, 2), dtype=torch.float64, device="cuda")


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    from xspde_matlab_b200 import _lib
    L = _lib.lib()
    path = _path(SMALL)
    nb = 2
    stream = torch.cuda.current_stream()
    for nc in (1, 2):
        ref = _av(path, nb)
        _lib.check(L.xs_run_path_device(path.h, 0, nb, nc, None, ctypes.c_void_p(ref.data_ptr()), None,
                                        ctypes.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize()
        scale = float(ref.abs().max())
        for _ in range(2):
            out = _av(path, nb)
            _lib.check(L.xs_run_path_device_noalloc(path.h, 0, nb, nc, ctypes.c_void_p(out.data_ptr()),
                                                    ctypes.c_void_p(stream.cuda_stream)))
            torch.cuda.synchronize()
            _lib.check(L.xs_sync(path.h))
            err = float((out - ref).abs().max()) / scale
            assert err < 1e-10, (nc, err)


def test_noalloc_refuses_launch_larger_than_scratch():
    import torch
    from xspde_matlab_b200 import _lib
    L = _lib.lib()
    big = dict(SMALL, points=[51, 64], ensembles=[1024, 8, 1], checks=0, observe=["@(a,p) a.*conj(a)"])
    path = _path(big)
    nb = 8
    av = _av(path, nb)
    stream = torch.cuda.current_stream()
    _lib.check(L.xs_run_path_device(path.h, 0, nb, 1, None, ctypes.c_void_p(av.data_ptr()), None,
                                    ctypes.c_void_p(stream.cuda_stream)))
    torch.cuda.synchronize()
    rc = L.xs_run_path_device_noalloc(path.h, 0, nb, 1, ctypes.c_void_p(av.data_ptr()),
                                      ctypes.c_void_p(stream.cuda_stream))
    assert rc == -1
    assert "fixed scratch holds 1048576" in _lib.last_error()


def test_noalloc_refuses_handles_it_cannot_serve():
    """The guards that keep the entry point from reading tables it does not
    have: a check pass the handle has not run yet (its propagator tables are
    missing: XS_ERR_ARG), a streaming-path handle and a handle whose field
    lives in device memory (both would need allocated buffers:
    XS_ERR_UNSUPPORTED)."""
    import torch
    from xspde_matlab_b200 import GpuPath, _lib, xpreferences
    L = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    path = _path(SMALL)
    av = _av(path, 1)
    _lib.check(L.xs_run_path_device(path.h, 0, 1, 1, None, ctypes.c_void_p(av.data_ptr()), None, stream))
    torch.cuda.synchronize()
    assert L.xs_run_path_device_noalloc(path.h, 0, 1, 2, ctypes.c_void_p(av.data_ptr()), stream) == -7
    assert "not prepared" in _lib.last_error()
    lattice = dict(dimensions=3, points=[3, 64, 64], ranges=[0.2, 10.0, 10.0], steps=2, ensembles=[2, 1, 1],
                   noises=2, method="MP", checks=0, deriv="@(a,w,p) -a + 0.01*w(1,:)", initial="@(v,p) 1 + 0*v(1,:)",
                   linear="@(p) 0.1i*(p.Dx.^2+p.Dy.^2)", observe=["@(a,p) abs(a).^2"])
    stream_path = GpuPath(xpreferences([lattice])[0], path_kind=2)
    assert L.xs_run_path_device_noalloc(stream_path.h, 0, 1, 1, ctypes.c_void_p(av.data_ptr()), stream) == -9
    assert "resident path only" in _lib.last_error()
    big = dict(lattice, points=[3, 128, 128], precision="fp64")
    gpath = GpuPath(xpreferences([big])[0], path_kind=1)
    assert L.xs_run_path_device_noalloc(gpath.h, 0, 1, 1, ctypes.c_void_p(av.data_ptr()), stream) == -9
    assert "shared memory" in _lib.last_error()
