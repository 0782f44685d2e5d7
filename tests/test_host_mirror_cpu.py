"""The host mirror of xsim/xensemble (xspde_matlab_b200.xsim) on CPU: its block
loop, moment sums, extrapolation, error columns, comparisons and axis handling
must reproduce the oracle's xsim when the device path is replaced by one that
returns the oracle's own block means (the device path itself is checked against
the same oracle by the GPU parity tests)."""
import warnings

import numpy as np
import pytest

from oracle import xspde_ref as X
from tests.gpu_util import oracle_block_av


class OraclePath:
    """Stands in for GpuPath: p.path of each block from the oracle's xpath."""

    def __init__(self, p, odict):
        self.p = p
        self.o = odict
        q = X.xpreferences([odict])[0]
        self.shapes = [tuple(s) for s in q.d_av]
        self.per_block = 2 * sum(int(np.prod(s)) for s in self.shapes)

    def av_shapes(self):
        return self.shapes

    def run_path(self, first, nblocks, nc, a_in=None, a_out=False, raw=False):
        av = []
        for b in range(first, first + nblocks):
            out = oracle_block_av(self.o, b, nc)
            av.append([np.asarray(x, dtype=complex).reshape(s, order="F") for x, s in zip(out[0], self.shapes)])
        return av, None


def _run(monkeypatch, g, o):
    import importlib
    M = importlib.import_module("xspde_matlab_b200.xsim")  # the module (the package exports a function xsim)
    monkeypatch.setattr(M, "GpuPath", lambda p, path_kind=0, runtime_params=False: OraclePath(p, o))
    eg, dg, _ = M.xsim(g)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        eo, do, _ = X.xsim(o)
    return np.asarray(eg), dg, np.asarray(eo), do


def _close(eg, dg, eo, do):
    # 1e-10: the mirror's moment sums are compensated, the oracle's plain (last-digit differences,
    # amplified by the cancellation in the sampling-error column)
    keep = [i for i in range(len(eo)) if i != 5]  # error(sx+2) with sx = 3 is the run time
    assert np.allclose(eg[keep], eo[keep], rtol=1e-10, atol=1e-15), (eg, eo)
    for a, b in zip(dg[0], do[0]):
        assert np.allclose(np.asarray(a), np.asarray(b), rtol=1e-10, atol=1e-13)


def test_mirror_matches_oracle_stochastic_spde_with_compare(monkeypatch):
    base = dict(dimensions=2, points=[7, 16], ranges=[1.0, 8.0], steps=2, ensembles=[4, 3, 2], noises=2,
                method="MP", checks=1, order=1)
    g = dict(base, deriv="@(a,w,p) 1i*a.*conj(a).*a - 0.1*a + 0.05*(w(1,:)+1i*w(2,:))",
             initial="@(v,p) exp(-p.x.^2) + 0.01*v(1,:)", linear="@(p) 1i*p.Dx.^2",
             observe=["@(a,p) a.*conj(a)", "@(a,p) Int(abs(a).^2, p)"],
             compare=[None, lambda p: np.sqrt(np.pi / 2) * np.exp(-0.2 * p.t)])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a - 0.1 * a + 0.05 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-p.x ** 2) + 0.01 * v[0:1], linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a), lambda a, p: X.Int(abs(a) ** 2, p)],
             compare=[None, lambda p: np.sqrt(np.pi / 2) * np.exp(-0.2 * p.t)])
    _close(*_run(monkeypatch, g, o))


@pytest.mark.parametrize("order", [0, 2])
def test_mirror_matches_oracle_kspace_and_spectrum(monkeypatch, order):
    """k-space axes (centred, p.kc) and a time spectrum (frequency axis), with and
    without Richardson extrapolation of the check passes."""
    base = dict(dimensions=2, points=[9, 16], ranges=[2.0, 8.0], steps=2, ensembles=[4, 2, 1], noises=2,
                method="RK4", checks=1, order=order, transforms=[[0, 1], [1, 0]])
    g = dict(base, deriv="@(a,w,p) -0.3*a + 0.1*(w(1,:)+1i*w(2,:))", initial="@(v,p) exp(-p.x.^2)",
             linear="@(p) 0.5i*p.Dx.^2", observe=["@(a,p) abs(a).^2", "@(a,p) abs(a).^2"])
    o = dict(base, deriv=lambda a, w, p: -0.3 * a + 0.1 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 0.5j * p.Dx ** 2,
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: abs(a) ** 2])
    _close(*_run(monkeypatch, g, o))


def _quantum():
    """Examples/SDE_1D/Quantum.m, shorter run: the oscillator driven by its input noise
    field, with the input and output fields as auxiliary cells and time spectra."""
    T = 40.0
    c = 2 * np.pi / T
    base = dict(points=[201], ranges=[T], order=2, auxfields=2, noises=2, ensembles=[100, 1, 12],
                transforms=[[1], [1], [1], [0]])
    g = dict(base, initial="@(w,p) (w(1,:)+1i*w(2,:))/2", deriv="@(a,w,p) -a(1,:)+sqrt(2)*(w(1,:)+1i*w(2,:))/2",
             define="@(a,w,p) [(w(1,:)+1i*w(2,:))/2; sqrt(2)*a(1,:)-(w(1,:)+1i*w(2,:))/2]",
             observe=["@(a,x,p) %r*abs(a(1,:)).^2" % c, "@(a,x,p) %r*abs(x(1,:)).^2" % c,
                      "@(a,x,p) %r*abs(x(2,:)).^2" % c, "@(a,x,p) abs(a(1,:)).^2"])

    def a1(w):
        return (w[0:1] + 1j * w[1:2]) / 2
    o = dict(base, initial=lambda w, p: a1(w), deriv=lambda a, w, p: -a[0:1] + np.sqrt(2) * a1(w),
             define=lambda a, w, p: np.concatenate([a1(w), np.sqrt(2) * a[0:1] - a1(w)]),
             observe=[lambda a, x, p: c * abs(a[0:1]) ** 2, lambda a, x, p: c * abs(x[0:1]) ** 2,
                      lambda a, x, p: c * abs(x[1:2]) ** 2, lambda a, x, p: abs(a[0:1]) ** 2])
    return g, o


class _CoarseUlpPath(OraclePath):
    """The oracle's blocks with the input-field spectrum of the coarse pass moved by a
    few units in the last place: the size of what a coarse noise formed with a fused
    multiply-add, (z2 s + round(z1 s)) / 2, instead of two rounded products gives."""

    def run_path(self, first, nblocks, nc, a_in=None, a_out=False, raw=False):
        av, _ = super().run_path(first, nblocks, nc, a_in, a_out, raw)
        if nc == 2:
            for row in av:
                row[1] = row[1] * (1 + 1e-15)
        return av, None


def test_mirror_quantum_step_error_counts_only_nonzero_observables(monkeypatch):
    """The input field x(1) = w/2 has the same time spectrum in both check passes: the
    coarse noise is the mean of the fine pass's two scaled draws bit for bit
    (Simulator/xnoise.m:32-35) and the fine pass records the mean of its half steps.
    Its step error is then exactly zero, and xsim.m's error vector averages the step
    errors over the observables above p.tol = 1e-20 only: three here.  A roundoff-sized
    difference between the passes makes it four, and the step-error entry falls by
    sqrt(3/4) with no visible change in any data column."""
    import importlib
    g, o = _quantum()
    eg, dg, eo, do = _run(monkeypatch, g, o)
    _close(eg, dg, eo, do)
    assert np.all(np.asarray(do[0][1])[:, 1] == 0)  # x(1) spectrum: zero step error
    assert np.all(np.asarray(dg[0][1])[:, 1] == 0)
    M = importlib.import_module("xspde_matlab_b200.xsim")
    monkeypatch.setattr(M, "GpuPath", lambda p, path_kind=0, runtime_params=False: _CoarseUlpPath(p, o))
    eu, du, _ = M.xsim(g)
    eu = np.asarray(eu)
    assert 0 < np.max(np.asarray(du[0][1])[:, 1]) < 1e-15
    assert np.isclose(eu[1], eo[1] * np.sqrt(3 / 4), rtol=1e-9)
    assert np.isclose(eu[2], eo[2], rtol=1e-12)
    for a, b in zip(du[0], do[0]):
        assert np.allclose(np.asarray(a)[:, 0], np.asarray(b)[:, 0], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("inp", [
    dict(dimensions=2, points=[7, 16], ranges=[1.0, 8.0], steps=2, noises=2, checks=1),
    dict(dimensions=3, points=[5, 12, 10], ranges=[0.5, 6.0, 4.0], steps=3, knoises=2, krandoms=1, checks=0),
    dict(points=[41], ranges=[8.0], auxfields=2, noises=2, transforms=[[1], [0]]),
    dict(dimensions=2, points=[9, 16], ranges=[2.0, 8.0], transforms=[0, 1], inrandoms=3),
])
def test_mirror_preferences_match_oracle(inp):
    """Derived constants of the host mirror's xpreferences (grids, k axes, noise
    scales, default noise and random counts, transform flags) equal the oracle's."""
    from xspde_matlab_b200.xsim import xpreferences as mirror
    q = mirror([dict(inp)])[0]
    r = X.xpreferences([dict(inp)])[0]
    assert q.points == r.points and q.steps[0] == r.steps[0] and q.checks[0] == r.checks[0]
    assert q.noises == r.noises and q.inrandoms == r.inrandoms
    assert q.knoises == r.knoises and q.krandoms == r.krandoms and q.auxfields == r.auxfields
    assert np.isclose(q.dt, r.dt) and np.allclose(q.dx, r.dx) and np.allclose(q.dk, r.dk)
    for d in range(len(q.kc)):
        assert np.allclose(q.kc[d], r.kc[d])
    assert [list(t) for t in q.transforms] == [list(t)[:len(q.transforms[0])] for t in r.transforms]


def test_mirror_matches_oracle_axes_and_cutoffs(monkeypatch):
    """Output axis selection (p.axes: all points, the middle point, the last point,
    explicit indices; Applications/SPDE/xcompress.m) and p.cutoffs."""
    base = dict(dimensions=3, points=[5, 8, 6], ranges=[0.5, 6.0, 4.0], steps=2, ensembles=[4, 2, 1], noises=2,
                method="MP", checks=1, order=1, axes=[None, [0, -1, 0], [0, [2, 5], -2]], cutoffs=[0.0, 0.1, 0.0])
    g = dict(base, deriv="@(a,w,p) -0.2*a + 0.1*w(1,:)", initial="@(v,p) exp(-(p.x.^2+p.y.^2)/4)",
             linear="@(p) 0.3i*(p.Dx.^2+p.Dy.^2)", observe=["@(a,p) abs(a).^2", "@(a,p) real(a)", "@(a,p) imag(a)"])
    o = dict(base, deriv=lambda a, w, p: -0.2 * a + 0.1 * w[0:1], initial=lambda v, p: np.exp(-(p.x ** 2 + p.y ** 2) / 4),
             linear=lambda p: 0.3j * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: np.real(a), lambda a, p: np.imag(a)])
    eg, dg, eo, do = _run(monkeypatch, g, o)
    for a, b in zip(dg[0], do[0]):
        assert np.shape(a) == np.shape(b)
    _close(eg, dg, eo, do)


def test_mirror_saves_matlab_file(monkeypatch, tmp_path):
    """p.file: error, data, input and raw in a MATLAB file (Simulator/xsim.m:207-210)."""
    import scipy.io
    base = dict(dimensions=2, points=[5, 8], ranges=[0.5, 4.0], steps=2, ensembles=[4, 2, 1], noises=2,
                method="MP", checks=1, order=1, file=str(tmp_path / "run.mat"))
    g = dict(base, deriv="@(a,w,p) -0.2*a + 0.1*w(1,:)", initial="@(v,p) exp(-p.x.^2)",
             linear="@(p) 0.3i*p.Dx.^2", observe=["@(a,p) abs(a).^2", "@(a,p) Int(abs(a).^2, p)"])
    o = dict(base, deriv=lambda a, w, p: -0.2 * a + 0.1 * w[0:1], initial=lambda v, p: np.exp(-p.x ** 2),
             linear=lambda p: 0.3j * p.Dx ** 2, observe=[lambda a, p: abs(a) ** 2, lambda a, p: X.Int(abs(a) ** 2, p)])
    eg, dg, eo, do = _run(monkeypatch, g, o)
    m = scipy.io.loadmat(str(tmp_path / "run.mat"))
    assert np.array_equal(m["error"][0], eg)
    for n in range(2):
        assert np.allclose(m["data"][0, 0][0, n], np.asarray(dg[0][n]))
    inp0 = m["input"][0, 0]
    assert list(inp0["points"][0, 0][0]) == [5, 8] and inp0["method"][0, 0][0] == "MP"


def test_save_mat_raw_cells(tmp_path):
    """raw{s, nc, k} is saved as a cell array of the trajectories' fields."""
    import scipy.io
    from xspde_matlab_b200.xsim import save_mat, xpreferences
    inp = xpreferences([dict(points=[3], ranges=[1.0], ensembles=[2, 2, 1])])
    r = [[[np.full((1, 3, 2), k + 10 * nc + 0.5j) for k in range(2)] for nc in range(2)]]
    save_mat(str(tmp_path / "raw.mat"), np.arange(6.0), [[np.ones((3, 3))]], inp, r)
    m = scipy.io.loadmat(str(tmp_path / "raw.mat"))
    assert m["raw"].shape == (1, 2, 2)
    assert np.allclose(m["raw"][0, 1, 1], 11 + 0.5j)
