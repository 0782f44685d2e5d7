"""The 3D streaming path (xs_stream3.cuh) against the FP64 oracle.

Lattices with a DST/DCT transform in every dimension and too large for shared
memory run as plane passes (T_y^-1, T_x^-1, the MP midpoint step with Philox
noise and the Dirichlet mask, T_x, T_y) and z-line passes (T_z, exp(L dt)^m,
T_z^-1) over a field in HBM.  The oracle (oracle/xspde_ref.py) restates
Simulator/xpath.m:29-86, Applications/SDE/MP.m:10-26 and
Applications/SPDE/xprop.m:18-42 with the reference's transforms
(Applications/SPDE/xdct1.m, xdst1.m, xdct2.m, xdct3.m, xdst2.m, xdst3.m).
Checked: block means of a site observable and of an Int over the lattice, the
final field, both check passes; every transform type in every position
(Neumann, Dirichlet and the two mixed ends), lattices that are not cubic, the
64^3 Allen-Cahn benchmark lattice in FP64 and in FP32 bulk, and a diverging
trajectory reported as XS_ERR_NAN.
"""
import numpy as np
import pytest

from oracle import xspde_ref as X
from tests.gpu_util import oracle_block_av, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-5


def _ac(points, boundaries, precision, checks=1, ens=(2, 2, 1), steps=2, ranges=(6.0, 5.0, 4.0)):
    """Stochastic Allen-Cahn with real noise and a random initial field (whose
    site values scale as 1/sqrt(dV): the lattice spacing must stay coarse
    enough for the cubic drift to stay finite)."""
    base = dict(dimensions=4, points=list(points), ranges=[0.01 * steps * (points[0] - 1)] + list(ranges),
                steps=steps, ensembles=list(ens), noises=1, inrandoms=1, method="MP", checks=checks,
                boundaries=[None] + [[list(b)] for b in boundaries])
    g = dict(base, precision=precision, deriv="@(a,w,p) a - a.^3 + 0.1*w(1,:)", initial="@(v,p) 0.3*v(1,:) + 0.5",
             linear="@(p) 0.05*(p.Dx.^2+p.Dy.^2+p.Dz.^2)",
             observe=["@(a,p) abs(a).^2", "@(a,p) Int(real(a).^2, p)"])
    o = dict(base, deriv=lambda a, w, p: a - a ** 3 + 0.1 * w[0:1], initial=lambda v, p: 0.3 * v[0:1] + 0.5,
             linear=lambda p: 0.05 * (p.Dx ** 2 + p.Dy ** 2 + p.Dz ** 2),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: X.Int(np.real(a) ** 2, p)])
    return g, o


def _run(g, blocks, nc, a_out=True):
    from xspde_matlab_b200 import GpuPath, xpreferences
    path = GpuPath(xpreferences([g])[0], path_kind=2)
    assert path.kind == 3  # plane and z-line passes
    return path.run_path(blocks[0], len(blocks), nc, a_out=a_out)


def _check(g, o, blocks, ncs, tol, fields=True):
    ens1 = g["ensembles"][0]
    for nc in ncs:
        av_g, a_g = _run(g, blocks, nc, a_out=fields)
        for i, b in enumerate(blocks):
            av_o, a_o = oracle_block_av(o, b, nc)
            for k in range(len(av_o)):
                e = rel_err(av_g[i][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
                # per output time, for the failure message
                et = [rel_err(av_g[i][k][:, n], av_o[k][:, n]) for n in range(av_o[k].shape[1])]
                assert e < tol, (nc, b, k, e, et)
            if fields:
                e = rel_err(a_g[..., ens1 * i:ens1 * (i + 1)], a_o)
                assert e < tol, (nc, b, "field", e)


@pytest.mark.parametrize("points,boundaries", [
    ((3, 32, 16, 24), ((-1, -1), (1, 1), (-1, 1))),   # DCT-I, DST-I (both folded), DCT-III/II
    ((3, 16, 32, 16), ((1, 1), (-1, 1), (1, -1))),    # DST-I, DCT-III/II, DST-III/II
    ((3, 24, 8, 32), ((-1, 1), (1, -1), (-1, -1))),   # mixed ends in x and y, DCT-I in z
])
def test_stream3_fp64_matches_oracle(points, boundaries):
    g, o = _ac(points, boundaries, "fp64")
    _check(g, o, [0, 1], [1, 2], FP64_TOL)


def test_stream3_64cube_fp64_matches_oracle():
    """The 3D benchmark lattice (64^3; Neumann x, Dirichlet y, Neumann-Dirichlet z)."""
    g, o = _ac((2, 64, 64, 64), ((-1, -1), (1, 1), (-1, 1)), "fp64", ens=(2, 1, 1), ranges=(20.0, 20.0, 20.0))
    _check(g, o, [1], [1, 2], FP64_TOL)


def test_stream3_64cube_fp32_each_observable_within_bound():
    """FP32 fields and matrices with FP64 propagator tables and moments: each
    observable within 1e-5 relative of the FP64 oracle."""
    g, o = _ac((2, 64, 64, 64), ((-1, -1), (1, 1), (-1, 1)), "fp32", ens=(2, 1, 1), checks=0, steps=3,
               ranges=(20.0, 20.0, 20.0))
    _check(g, o, [0], [1], FP32_TOL, fields=False)


def test_stream3_diverging_trajectory_reports_nan():
    from xspde_matlab_b200 import GpuPath, _lib, xpreferences
    g, _ = _ac((3, 32, 16, 24), ((-1, -1), (1, 1), (-1, 1)), "fp64", checks=0)
    g.update(deriv="@(a,w,p) a.^3", initial="@(v,p) 40 + 0*v(1,:)", ranges=[2.0, 6.0, 5.0, 4.0])
    path = GpuPath(xpreferences([g])[0], path_kind=2)
    assert path.kind == 3
    with pytest.raises(_lib.XsError) as err:
        path.run_path(0, 1, 1, a_out=True)
    assert err.value.code == -5  # XS_ERR_NAN


@pytest.mark.parametrize("boundaries", [
    ((-1, -1), (1, 1), (-1, 1)),   # DCT-I in x, DST-I in y (the benchmark's boundaries)
    ((1, -1), (-1, 1), (1, 1)),    # DST-III/II in x, DCT-III/II in y
])
def test_stream3_tensor_core_plane_pass_fp32(boundaries, monkeypatch):
    """64 x 64 planes in FP32 take the tensor-core plane pass (xs_stream3_tc.cuh:
    the four transforms as tcgen05 TF32 GEMMs with the three-term split): both
    check passes, each observable and the final field within 1e-5 of the FP64
    oracle, like the CUDA-core pass (XSPDE_B200_TC3=0); the two passes round
    differently, so their results are not bit-identical."""
    g, o = _ac((2, 64, 64, 8), boundaries, "fp32", ens=(2, 1, 1), steps=3, ranges=(20.0, 20.0, 5.0))
    _check(g, o, [0], [1, 2], FP32_TOL)
    av_tc, a_tc = _run(g, [0], 1)
    monkeypatch.setenv("XSPDE_B200_TC3", "0")
    av_cc, a_cc = _run(g, [0], 1)
    assert rel_err(a_tc, a_cc) < 2 * FP32_TOL
    assert not np.array_equal(a_tc, a_cc)
