"""The MATLAB MEX binding (xspde_matlab_b200/mex/xspde_path_mex.c), without MATLAB.

The binding maps xSPDE's p.path hook (Simulator/xpath.m:1, called at
Simulator/xensemble.m:79) onto xs_run_path_raw.  MATLAB is not installed
here, so the tests compile it with gcc against a stand-in of the MEX API
(tests/mex_stub/mex.h, fake_mex.c) and a driver that builds the parameter
struct the way xpreferences lays it out (cells for fields, noises, points,
the function handles and boundaries; d.av; a named scalar) and seeds the
generator the way xensemble does:
  - CPU: the binding, the stand-in and the driver compile and link against
    libxspde_b200.so with -Wall -Werror.
  - GPU: the outputs of one p.path call through the binding -- block means
    av{o} in the dimensions p.d.av{o}, the final field and raw{1} -- equal
    those of the Python host's GpuPath.run_path for the same block, check
    pass and initial field, both check passes; the block comes from the seed
    xensemble sets, nsp = p.seed + npar + (j-1) ensembles(3).
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STUB = os.path.join(ROOT, "tests", "mex_stub")
LIBDIR = os.path.join(ROOT, "xspde_matlab_b200")


def _build(out_dir):
    exe = os.path.join(out_dir, "run_path_mex")
    cmd = ["gcc", "-std=c11", "-O1", "-Wall", "-Werror", "-Wno-unused-function", "-I", STUB,
           "-I", os.path.join(ROOT, "include"),
           os.path.join(LIBDIR, "mex", "xspde_path_mex.c"), os.path.join(STUB, "fake_mex.c"),
           os.path.join(STUB, "run_path_mex.c"), "-L", LIBDIR, "-lxspde_b200", "-Wl,-rpath," + LIBDIR, "-lm",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_mex_binding_compiles_against_the_mex_api(tmp_path):
    exe = _build(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [1, 2])
def test_mex_binding_matches_python_host_path(tmp_path, nc):
    from xspde_matlab_b200 import GpuPath, xpreferences
    exe = _build(str(tmp_path))
    x = -5.0 + 10.0 / 31 * np.arange(32)
    rs = np.random.default_rng(3)
    a_in = (np.exp(-x ** 2)[None, :, None] + 0.01 * rs.standard_normal((1, 32, 4))).astype(np.complex128)
    fin = tmp_path / "a_in.bin"
    fin.write_bytes(np.asfortranarray(a_in).ravel(order="F").tobytes())
    fout = tmp_path / "out.bin"
    block = 1
    r = subprocess.run([exe, str(fin), str(block), str(nc), str(fout)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    data = fout.read_bytes()
    dims = np.frombuffer(data[-64:], dtype=np.int64)
    vals = np.frombuffer(data[:-64], dtype=np.complex128)
    n_av, n_a, n_raw = 5 * 32, 32 * 4, 5 * 32 * 4
    av1, av2 = vals[:n_av], vals[n_av:2 * n_av]
    a_fin = vals[2 * n_av:2 * n_av + n_a]
    raw1 = vals[2 * n_av + n_a:2 * n_av + n_a + n_raw]
    assert list(dims[:4]) == [1, n_av, 1, n_raw]
    p = xpreferences([dict(dimensions=2, points=[5, 32], ranges=[0.5, 10.0], steps=2, checks=1, ensembles=[4, 2, 1],
                           noises=2, method="MP", seed=7, rawdata=1, params={"g": 0.01},
                           deriv="@(a,w,p) 1i*a.*conj(a).*a + p.g*(w(1,:)+1i*w(2,:))/sqrt(2)",
                           initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2",
                           observe=["@(a,p) a.*conj(a)", "@(a,p) real(a)"])])[0]
    av, a_out, rw = GpuPath(p).run_path(block, 1, nc, a_in=a_in, a_out=True, raw=True)
    for got, want in ((av1, av[0][0]), (av2, av[0][1]), (a_fin, a_out), (raw1, rw)):
        want = np.asarray(want).ravel(order="F")
        assert np.allclose(got, want, rtol=1e-12, atol=1e-14)
