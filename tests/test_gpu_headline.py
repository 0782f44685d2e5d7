"""GPU parity at the benchmark configurations' own sizes.

The 2D benchmark problem (256x256 periodic GPE/CGL, MP) runs on the streaming
kernels (x-row pass with a 256-point register four-step FFT, y-column pass),
so it is checked here at 256x256, not only at a reduced lattice:
  - FP64 fields: block-mean observables <|a|^2>(x,y,t), <Re a>(x,y,t) and the
    final field agree with the FP64 oracle (oracle/xspde_ref.py, the
    restatement of Simulator/xpath.m:29-86 and Applications/SDE/MP.m:10-26)
    to 1e-10 relative to the largest |value|, for both step-halving passes.
  - FP32 fields with FP64 propagator tables and moments: each observable
    within 1e-5 relative of the FP64 oracle (the bound stated for the FP32
    bulk mode).
The 1D benchmark problem (stochastic NLS, 64 points, 51 x 4 steps, 1024
trajectories in 8 blocks) runs at its full size through the resident kernel,
RK4 and MP, every block against the oracle.
"""
import numpy as np
import pytest

from tests.gpu_util import oracle_block_av, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-5


def _gpe_256(precision, checks=1, ens=(2, 2, 1), points=3, method="MP"):
    """The benchmark's 256x256 problem with the benchmark's step (dtr = 0.01)
    over a shorter time: `points` output times, 10 steps between them."""
    base = dict(dimensions=3, points=[points, 256, 256], ranges=[0.1 * (points - 1), 20.0, 20.0], steps=10,
                ensembles=list(ens), noises=2, method=method, checks=checks)
    g = dict(base, precision=precision,
             deriv="@(a,w,p) (1-abs(a).^2).*a - 0.5i*abs(a).^2.*a + 0.05*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) 1 + 0.1*(v(1,:)+1i*v(2,:))/sqrt(2)", linear="@(p) (1i+0.1)*(p.Dx.^2+p.Dy.^2)",
             observe=["@(a,p) abs(a).^2", "@(a,p) real(a)"])
    o = dict(base, deriv=lambda a, w, p: (1 - abs(a) ** 2) * a - 0.5j * abs(a) ** 2 * a
             + 0.05 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: 1 + 0.1 * (v[0:1] + 1j * v[1:2]) / np.sqrt(2),
             linear=lambda p: (1j + 0.1) * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: np.real(a)])
    return g, o


def _stream(g, blocks, nc, a_out=True):
    from xspde_matlab_b200 import GpuPath, xpreferences
    path = GpuPath(xpreferences([g])[0], path_kind=2)
    return path.run_path(blocks[0], len(blocks), nc, a_out=a_out)


def _check_blocks(av_g, a_g, o, blocks, nc, tol, ens1):
    worst = {}
    for i, b in enumerate(blocks):
        av_o, a_o = oracle_block_av(o, b, nc)
        for k in range(len(av_o)):
            e = rel_err(av_g[i][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
            worst[k] = max(worst.get(k, 0.0), e)
            assert e < tol, (nc, b, k, e)
        if a_g is not None:
            e = rel_err(a_g[..., ens1 * i:ens1 * (i + 1)], a_o)
            worst["field"] = max(worst.get("field", 0.0), e)
            assert e < tol, (nc, b, "field", e)
    return worst


@pytest.mark.parametrize("nc", [1, 2])
def test_gpe_256x256_streaming_fp64_matches_oracle(nc):
    """Both passes of a step-halving run (nc = 1 fine, nc = 2 coarse, whose
    noise is the mean of two fine draws, Simulator/xnoise.m:33-35)."""
    g, o = _gpe_256("fp64")
    av_g, a_g = _stream(g, [0, 1], nc)
    _check_blocks(av_g, a_g, o, [0, 1], nc, FP64_TOL, 2)


@pytest.mark.parametrize("nc", [1, 2])
def test_gpe_256x256_streaming_fp32_each_observable_within_bound(nc):
    """FP32 bulk (fields, FFTs, drift) with FP64 phase tables and moments:
    <|a|^2> and <Re a> each within 1e-5 relative of the FP64 oracle."""
    g, o = _gpe_256("fp32")
    av_g, _ = _stream(g, [0, 1], nc, a_out=False)
    worst = _check_blocks(av_g, None, o, [0, 1], nc, FP32_TOL, 2)
    assert set(worst) == {0, 1}


def test_gpe_256x256_streaming_fp64_longer_path():
    """Eleven output times (109 MP steps, one observation every 10 steps) of
    one block of two trajectories, no step halving."""
    g, o = _gpe_256("fp64", checks=0, ens=(2, 1, 1), points=11)
    av_g, a_g = _stream(g, [3], 1)
    _check_blocks(av_g, a_g, o, [3], 1, FP64_TOL, 2)


@pytest.mark.parametrize("nc", [1, 2])
def test_gpe_256x256_streaming_rk4_fp64_matches_oracle(nc):
    """RK4 (the reference's default deterministic stepper, Applications/SDE/RK4.m:7-42)
    on the 256x256 streaming path: both check passes, observables and final field."""
    g, o = _gpe_256("fp64", method="RK4")
    av_g, a_g = _stream(g, [0, 1], nc)
    _check_blocks(av_g, a_g, o, [0, 1], nc, FP64_TOL, 2)


SNLS_FULL = dict(dimensions=2, points=[51, 64], ranges=[1.0, 10.0], steps=4, ensembles=[128, 8, 1], noises=2)


def _snls_full(method, checks, precision):
    g = dict(SNLS_FULL, method=method, checks=checks, precision=precision,
             deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2",
             observe=["@(a,p) a.*conj(a)", "@(a,p) real(a)"])
    o = dict(SNLS_FULL, method=method, checks=checks,
             deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.01 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a), lambda a, p: np.real(a)])
    return g, o


@pytest.mark.parametrize("method,checks,precision,tol", [
    ("RK4", 0, "fp64", FP64_TOL), ("MP", 1, "fp64", FP64_TOL), ("RK4", 0, "fp32", FP32_TOL)])
def test_snls_1d_full_size_matches_oracle(method, checks, precision, tol):
    """64 points, 51 output times x 4 steps (200 steps to t = 1), 1024
    trajectories in 8 blocks: every block and every check pass."""
    from xspde_matlab_b200 import GpuPath, xpreferences
    g, o = _snls_full(method, checks, precision)
    path = GpuPath(xpreferences([g])[0])
    blocks = list(range(8))
    for nc in ([1, 2] if checks else [1]):
        av_g, a_g = path.run_path(0, 8, nc, a_out=True)
        _check_blocks(av_g, a_g if precision == "fp64" else None, o, blocks, nc, tol, 128)
