"""GPU parity of the streaming (HBM row/column pass) path against the oracle.

A 64x64 periodic lattice is forced onto the streaming kernels (path_kind=2):
the same x-row / y-column passes and FFT code that the 256x256 benchmark
uses, at a size the oracle finishes in seconds.  FP64 tolerance 1e-10
relative to max |av|; FP32 (FP64 propagator table, FP64 moments) 2e-4.
"""
import numpy as np
import pytest

from oracle import xspde_ref as X
from tests.gpu_util import oracle_block_av, rel_err

pytestmark = pytest.mark.gpu


def _case(checks, precision="fp64", points=(5, 64, 64), ens=(4, 2, 1), obs_int=True, method="MP"):
    base = dict(dimensions=3, points=list(points), ranges=[0.2, 12.0, 10.0], steps=2, ensembles=list(ens), noises=2,
                method=method, checks=checks)
    gobs = ["@(a,p) abs(a).^2", "@(a,p) real(a)"]
    oobs = [lambda a, p: abs(a) ** 2, lambda a, p: np.real(a)]
    if obs_int:
        gobs.append("@(a,p) Int(abs(a).^2, p.dx, [0 0; -2 3; -1 2], p)")
        oobs.append(lambda a, p: X.Int(abs(a) ** 2, p.dx, [[0, 0], [-2, 3], [-1, 2]], p))
    g = dict(base, precision=precision,
             deriv="@(a,w,p) (1-abs(a).^2).*a - 0.5i*abs(a).^2.*a + 0.05*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) 1 + 0.1*(v(1,:)+1i*v(2,:))/sqrt(2) + 0.2*exp(-p.x.^2-p.y.^2)",
             linear="@(p) (1i+0.1)*(p.Dx.^2+p.Dy.^2)", observe=gobs)
    o = dict(base, deriv=lambda a, w, p: (1 - abs(a) ** 2) * a - 0.5j * abs(a) ** 2 * a
             + 0.05 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: 1 + 0.1 * (v[0:1] + 1j * v[1:2]) / np.sqrt(2) + 0.2 * np.exp(-p.x ** 2 - p.y ** 2),
             linear=lambda p: (1j + 0.1) * (p.Dx ** 2 + p.Dy ** 2), observe=oobs)
    return g, o


def _run(g, blocks, nc, a_in=None, a_out=False):
    from xspde_matlab_b200 import GpuPath, xpreferences
    path = GpuPath(xpreferences([g])[0], path_kind=2)
    return path.run_path(blocks[0], len(blocks), nc, a_in=a_in, a_out=a_out)


@pytest.mark.parametrize("checks", [0, 1])
def test_stream_fp64_matches_oracle(checks):
    g, o = _case(checks)
    for nc in ([1, 2] if checks else [1]):
        av_g, _ = _run(g, [0, 1], nc)
        for i, b in enumerate([0, 1]):
            av_o, _ = oracle_block_av(o, b, nc)
            for k in range(len(av_o)):
                e = rel_err(av_g[i][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
                assert e < 1e-10, (nc, b, k, e)


def test_stream_fp32_bound():
    g, o = _case(1, precision="fp32")
    for nc in (1, 2):
        av_g, _ = _run(g, [1], nc)
        av_o, _ = oracle_block_av(o, 1, nc)
        for k in range(len(av_o)):
            e = rel_err(av_g[0][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
            assert e < 2e-4, (nc, k, e)


def test_stream_final_field_and_rectangular_lattice():
    g, o = _case(0, points=(4, 64, 256), ens=(2, 1, 1), obs_int=False)
    av_o, b_o = oracle_block_av(o, 0, 1)
    av_g, a_g = _run(g, [0], 1, a_out=True)
    assert rel_err(a_g, b_o) < 1e-10
    assert rel_err(av_g[0][0], av_o[0]) < 1e-10


@pytest.mark.parametrize("checks", [0, 1])
def test_stream_512_trajectories_final_field_match_oracle(checks):
    """512 trajectories in 2 blocks of 256 (the benchmark's block size) with
    the final field requested: FP64 observables and fields agree with the
    oracle for both blocks and both check passes."""
    g, o = _case(checks, points=(3, 64, 64), ens=(256, 2, 1))
    for nc in ([1, 2] if checks else [1]):
        av_g, a_g = _run(g, [0, 1], nc, a_out=True)
        for i, b in enumerate([0, 1]):
            av_o, a_o = oracle_block_av(o, b, nc)
            for k in range(len(av_o)):
                e = rel_err(av_g[i][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
                assert e < 1e-10, (nc, b, k, e)
            e = rel_err(a_g[..., 256 * i:256 * (i + 1)], a_o)
            assert e < 1e-10, (nc, b, "field", e)


def test_stream_nonseparable_linear_fp64():
    """A linear operator with a kx^2 ky^2 cross term is not separable, so the
    column pass reads the full [ky][kx] propagator table (the separable GPE
    operator above uses two 1D tables); both agree with the oracle."""
    g, o = _case(0, obs_int=False)
    g = dict(g, linear="@(p) (1i+0.1)*(p.Dx.^2+p.Dy.^2) + 0.02i*p.Dx.^2.*p.Dy.^2")
    o = dict(o, linear=lambda p: (1j + 0.1) * (p.Dx ** 2 + p.Dy ** 2) + 0.02j * p.Dx ** 2 * p.Dy ** 2)
    av_g, _ = _run(g, [0, 1], 1)
    for i, b in enumerate([0, 1]):
        av_o, _ = oracle_block_av(o, b, 1)
        for k in range(len(av_o)):
            e = rel_err(av_g[i][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
            assert e < 1e-10, (b, k, e)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_stream_tma_column_pass_bit_identical(precision, monkeypatch):
    """The column pass fed by TMA bulk tensor copies (XSPDE_B200_TMA=1, NY <= 256)
    and the plain one (default) do the same arithmetic: identical bits."""
    from xspde_matlab_b200 import GpuPath, xpreferences
    g, _ = _case(0, precision=precision, ens=(32, 2, 1))
    p = xpreferences([g])[0]
    monkeypatch.delenv("XSPDE_B200_TMA", raising=False)
    av_plain, a_plain = GpuPath(p, path_kind=2).run_path(0, 2, 1, a_out=True)
    monkeypatch.setenv("XSPDE_B200_TMA", "1")
    av_tma, a_tma = GpuPath(p, path_kind=2).run_path(0, 2, 1, a_out=True)
    assert np.array_equal(a_plain, a_tma)
    for b in range(2):
        for k in range(len(av_plain[b])):
            assert np.array_equal(av_plain[b][k], av_tma[b][k]), (b, k)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_stream_fused_halves_bit_identical(precision, monkeypatch):
    """With an even number of blocks the two halves of the trajectories run one
    pass apart and each row pass shares an xs_rc_pass launch with the other
    half's column pass; per trajectory the arithmetic is unchanged, so fields,
    site observables and Int reductions equal the one-pass-at-a-time schedule
    (the default) bit for bit, for both check passes (XSPDE_B200_FUSE=1 selects it)."""
    import ctypes
    from xspde_matlab_b200 import GpuPath, _lib, xpreferences
    g, _ = _case(1, precision=precision, ens=(8, 4, 1))
    p = xpreferences([g])[0]
    L = _lib.lib()
    n = len(_lib.KERNEL_KINDS)
    for nc in (1, 2):
        monkeypatch.delenv("XSPDE_B200_FUSE", raising=False)
        av_a, a_a = GpuPath(p, path_kind=2).run_path(0, 4, nc, a_out=True)
        monkeypatch.setenv("XSPDE_B200_FUSE", "1")
        path = GpuPath(p, path_kind=2)
        _lib.check(L.xs_set_kernel_timing(path.h, 1))
        av_b, a_b = path.run_path(0, 4, nc, a_out=True)
        kms, kl = (ctypes.c_double * n)(), (ctypes.c_longlong * n)()
        _lib.check(L.xs_kernel_stats(path.h, 1, kms, kl))
        assert kl[_lib.KERNEL_KINDS.index("rc_pass")] > 0
        assert np.array_equal(a_a, a_b), nc
        for b in range(4):
            for k in range(len(av_a[b])):
                assert np.array_equal(av_a[b][k], av_b[b][k]), (nc, b, k)


@pytest.mark.parametrize("checks", [0, 1])
def test_stream_rk4_fp64_matches_oracle(checks):
    """RK4 on the streaming kernels (Applications/SDE/RK4.m:7-42): two fields in HBM,
    three row passes and column passes on both fields per step, one noise for all
    stages; block means and the final field against the oracle at 1e-10, both
    check passes (the coarse pass averages two fine draws)."""
    g, o = _case(checks, method="RK4")
    for nc in ([1, 2] if checks else [1]):
        av_g, a_g = _run(g, [0, 1], nc, a_out=True)
        for i, b in enumerate([0, 1]):
            av_o, a_o = oracle_block_av(o, b, nc)
            for k in range(len(av_o)):
                e = rel_err(av_g[i][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
                assert e < 1e-10, (nc, b, k, e)
            e = rel_err(a_g[..., 4 * i:4 * (i + 1)], a_o)
            assert e < 1e-10, (nc, b, "field", e)


def test_stream_rk4_fp32_bound():
    g, o = _case(1, precision="fp32", method="RK4")
    for nc in (1, 2):
        av_g, _ = _run(g, [1], nc)
        av_o, _ = oracle_block_av(o, 1, nc)
        for k in range(len(av_o)):
            e = rel_err(av_g[0][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
            assert e < 2e-4, (nc, k, e)


def test_stream_rk4_single_output_time_every_step_observed():
    """steps = 1: every step is followed by an observation, so no pass 3 is fused
    with the next step's pass 1; with steps = 2 (above) every other one is."""
    g, o = _case(0, points=(4, 64, 64), method="RK4", obs_int=False)
    g = dict(g, steps=1)
    o = dict(o, steps=1)
    av_g, a_g = _run(g, [0], 1, a_out=True)
    av_o, a_o = oracle_block_av(o, 0, 1)
    assert rel_err(a_g, a_o) < 1e-10
    for k in range(len(av_o)):
        assert rel_err(av_g[0][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F")) < 1e-10


def test_stream_host_copies_overlapped_equal_single_block_calls():
    """xs_run_path on the streaming path with a host initial field runs its blocks in
    groups, copying the next group's field in and the previous group's means out
    while a group integrates; every trajectory does the same arithmetic as in a
    call for its block alone, so block means and final fields are bit-identical."""
    from xspde_matlab_b200 import GpuPath, xpreferences
    g, _ = _case(1, ens=(8, 4, 1))
    path = GpuPath(xpreferences([g])[0], path_kind=2)
    rs = np.random.default_rng(11)
    a_in = (1 + 0.1 * rs.standard_normal((1, 64, 64, 32)) + 0.1j * rs.standard_normal((1, 64, 64, 32)))
    for nc in (1, 2):
        av_all, a_all = path.run_path(0, 4, nc, a_in=a_in, a_out=True)
        for b in range(4):
            av_b, a_b = path.run_path(b, 1, nc, a_in=a_in[..., 8 * b:8 * (b + 1)], a_out=True)
            assert np.array_equal(a_all[..., 8 * b:8 * (b + 1)], a_b), (nc, b)
            for k in range(len(av_b[0])):
                assert np.array_equal(av_all[b][k], av_b[0][k]), (nc, b, k)
