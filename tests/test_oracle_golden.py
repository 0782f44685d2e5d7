"""Pin the CPU oracle against the reference's own golden values.

Examples/Batchtest.m:67-75 records the expected total RMS error e(1) of each
example project and accepts a result within a factor 1.001
(Examples/Batchtest.m:81).  The deterministic projects below do not depend on
MATLAB's random stream, so the oracle must reproduce them.
"""
import warnings

import numpy as np
import pytest

from oracle import philox
from oracle import xspde_ref as X
from tests.oracle_examples import DETERMINISTIC


@pytest.mark.parametrize("name", sorted(DETERMINISTIC))
def test_batchtest_deterministic_rows(name, golden_expected):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        e, data, inp = X.xsim(*DETERMINISTIC[name]())
    exp = golden_expected[name]
    assert exp / 1.001 < e[0] < exp * 1.001, (name, e[0], exp)


def test_philox_known_answers():
    # Published Philox4x32-10 known-answer vectors (Salmon et al., SC'11).
    kat = [((0, 0, 0, 0, 0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 6, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344, 0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for (c0, c1, c2, c3, k0, k1), want in kat:
        got = philox.philox4x32_10(c0, c1, c2, c3, k0, k1)
        assert tuple(int(x) for x in got) == want


def test_philox_normals_moments():
    z = philox.normals(4, 4096, 64, 3, 7, 11)
    assert abs(z.mean()) < 0.01
    assert abs(z.var() - 1) < 0.01
    assert abs(np.mean(z ** 4) - 3) < 0.05


def test_time_spectrum_exact_geometric_series():
    """p.transforms{n}(1) (Simulator/xpath.m:90-106): a linear ODE stepped by RK4 is
    a_j = r^j with r the RK4 amplification 1 + z + z^2/2 + z^3/6 + z^4/24, z = lambda dtr,
    so the recorded spectrum fsc/Nt sum_j r^j exp(2 pi i m j / Nt) at m = n - floor(P1/2)
    has the closed form fsc/Nt (1 - (r q)^Nt) / (1 - r q), q = exp(2 pi i m / Nt)."""
    lam = 2j - 0.3
    o = dict(dimensions=1, points=[33], ranges=[20.0], steps=4, ensembles=[2, 1, 1], noises=1, method="RK4",
             checks=0, deriv=lambda a, w, p: lam * a, initial=lambda v, p: 1 + 0 * v,
             observe=[lambda a, p: a, lambda a, p: a], transforms=[[1], [0]])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        e, data, inp = X.xsim(o)
    p = inp[0]
    P1, S = 33, 4
    nt = P1 * S
    dt = 20.0 / (P1 - 1)
    z = lam * dt / S
    r = 1 + z + z ** 2 / 2 + z ** 3 / 6 + z ** 4 / 24
    dw = 2 * np.pi / (20.0 + dt)
    fsc = np.sqrt(2 * np.pi) / dw
    m = np.arange(P1) - P1 // 2
    q = np.exp(2j * np.pi * m / nt)
    want = fsc / nt * (1 - (r * q) ** nt) / (1 - r * q)
    got = data[0][0][:, 0]
    assert np.max(np.abs(got - np.real(want))) < 1e-11 * np.max(np.abs(want))
    assert np.allclose(p.kc[0], m * dw)
    assert np.allclose(data[0][1][:, 0], np.real(r ** (S * np.arange(P1))), atol=1e-12)


def test_time_spectrum_equilibrium_known_answer():
    """Examples/SDE_1D/Equilibrium.m: the Ornstein-Uhlenbeck spectrum |a(w)|^2 equals
    its comparison T / (pi (1 + w^2)) within the sampling error, and |a(t)|^2 = 1."""
    o = dict(points=[200], steps=2, ranges=[25.0], seed=241, noises=2, ensembles=[50, 1, 12],
             initial=lambda w, p: (w[0] + 1j * w[1]) / np.sqrt(2), deriv=lambda a, w, p: -a + w[0] + 1j * w[1],
             observe=[lambda a, p: a * np.conj(a), lambda a, p: a * np.conj(a)], transforms=[[0], [1]])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        e, data, inp = X.xsim(o)
    w = inp[0].kc[0]
    spec, err = np.real(data[0][1][:, 0]), np.real(data[0][1][:, 2])
    exact = 25.0 / (np.pi * (1 + w ** 2))
    sel = np.abs(w) < 4
    assert np.all(np.abs(spec[sel] - exact[sel]) < 5 * err[sel] + 0.02 * exact[sel])
    tdom = np.real(data[0][0][:, 0])
    assert np.all(np.abs(tdom - 1) < 5 * np.real(data[0][0][:, 2]) + 0.02)


def _planar_init(u, v, p):
    return np.concatenate([(u[0:1] + 1j * u[1:2]) / np.sqrt(2), (v[0:1] + 1j * v[1:2]) / np.sqrt(2)], axis=0)


def _planar_deriv(a, w, z, p):
    return np.concatenate([(w[0:1] + 1j * w[1:2]) / np.sqrt(2), (z[0:1] + 1j * z[1:2]) / np.sqrt(2)], axis=0)


def test_knoise_planar_known_answer():
    """Examples/SPDE_3D/Planar.m on a smaller lattice: x-space noise drives a_1 and
    k-filtered noise (knoises, krandoms; Simulator/xnoise.m:39-50, xrandom.m:24-29)
    drives a_2; both integrals grow as the example's comparison (1 + t) nspace, and
    the k-space integral of |a_2(k)|^2 dk equals the x-space one (Parseval)."""
    o = dict(dimensions=3, fields=2, ranges=[1, 5, 5], points=[11, 16, 12], steps=2, noises=2, knoises=2,
             inrandoms=2, krandoms=2, ensembles=[10, 2, 6], initial=_planar_init, deriv=_planar_deriv,
             linear=lambda p: 0.5j * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: X.Int(a[0:1] * np.conj(a[0:1]), p),
                      lambda a, p: X.Int(a[1:2] * np.conj(a[1:2]), p.dk, p),
                      lambda a, p: X.Int(a[1:2] * np.conj(a[1:2]), p)],
             transforms=[[0, 0, 0], [0, 1, 1], [0, 0, 0]])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        e, data, inp = X.xsim(o)
    p = inp[0]
    t = p.xc[0]
    exact = (1 + t) * p.nspace
    for k in range(3):
        mean, err = np.real(data[0][k][:, 0]), np.real(data[0][k][:, 2])
        assert np.all(np.abs(mean - exact) < 5 * err + 1e-9 * exact), k
    assert np.allclose(data[0][1][:, 0], data[0][2][:, 0], rtol=1e-10)


def test_auxiliary_fields_quantum_known_answer():
    """Examples/SDE_1D/Quantum.m (shorter run): auxiliary fields from p.define
    (xpath.m:36-45, xensemble.m:74-77) carry the input and output fields of a
    damped oscillator; their spectra are flat at 1/2 and the oscillator's is
    1/(1 + w^2), the example's comparisons, within five sampling errors."""
    T = 40.0

    def a1(w):
        return (w[0:1] + 1j * w[1:2]) / 2
    o = dict(points=[201], ranges=[T], order=2, auxfields=2, noises=2, ensembles=[100, 1, 12],
             initial=lambda w, p: (w[0:1] + 1j * w[1:2]) / 2,
             deriv=lambda a, w, p: -a[0:1] + np.sqrt(2) * a1(w),
             define=lambda a, w, p: np.concatenate([a1(w), np.sqrt(2) * a[0:1] - a1(w)]),
             observe=[lambda a, x, p: (2 * np.pi / T) * abs(a[0:1]) ** 2,
                      lambda a, x, p: (2 * np.pi / T) * abs(x[0:1]) ** 2,
                      lambda a, x, p: (2 * np.pi / T) * abs(x[1:2]) ** 2, lambda a, x, p: abs(a[0:1]) ** 2],
             transforms=[[1], [1], [1], [0]])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        e, data, inp = X.xsim(o)
    w = inp[0].kc[0]
    sel = np.abs(w) < 3
    for k, exact in ((0, 1 / (1 + w ** 2)), (1, 0.5 + 0 * w), (2, 0.5 + 0 * w), (3, None)):
        mean, err = np.real(data[0][k][:, 0]), np.real(data[0][k][:, 2])
        if exact is None:
            assert np.all(np.abs(mean - 0.5) < 5 * err + 0.02)
        else:
            assert np.all(np.abs(mean[sel] - exact[sel]) < 5 * err[sel] + 1e-3), k


def _stat_check(data, o, exact, k=3.0):
    """Each point of the fine mean within 5 sampling errors + k step errors + 1e-3 of the exact."""
    d = np.real(data)
    mean, step, samp = d[:, 0], d[:, 1], d[:, 2]
    assert np.all(np.abs(mean - exact) < 5 * samp + k * step + 1e-3), (o, np.max(np.abs(mean - exact)))


def test_statistical_pins_kubo2_gain_wiener():
    """The reference examples' comparisons, which hold for any random-number stream:
    Examples/SDE_1D/Kubo2.m (RK2, <Re a> = exp(-t/2), <|a|^2> = 1), Gain.m (<|a|^2> = 1)
    and Wiener.m (Euler; <a>, <a^2>, <a^3>, <a^4> = 0, 4 + t, 0, 3 (4 + t)^2)."""
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        kubo = dict(ensembles=[400, 10], method="RK2", steps=5, initial=lambda w, p: 1 + 0 * w,
                    deriv=lambda a, w, p: 1j * w * a,
                    observe=[lambda a, p: np.real(a[0:1]), lambda a, p: a[0:1] * np.conj(a[0:1])])
        e, d, inp = X.xsim(kubo)
        t = inp[0].xc[0]
        _stat_check(d[0][0], "kubo <a>", np.exp(-t / 2))
        _stat_check(d[0][1], "kubo |a|^2", 1 + 0 * t)
        gain = dict(ranges=[4.0], noises=2, ensembles=[2000, 1, 10],
                    initial=lambda w, p: (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
                    deriv=lambda a, w, p: -a + w[0:1] + 1j * w[1:2], observe=[lambda a, p: a * np.conj(a)])
        e, d, inp = X.xsim(gain)
        _stat_check(d[0][0], "gain", 1 + 0 * inp[0].xc[0])
        wiener = dict(method="Euler", noises=1, ensembles=[250, 4, 10], initial=lambda v, p: 2 * v,
                      deriv=lambda a, w, p: w, observe=[lambda a, p: np.concatenate([a, a ** 2, a ** 3, a ** 4])])
        e, d, inp = X.xsim(wiener)
        t = inp[0].xc[0]
        m = np.reshape(np.real(d[0][0]), (4, len(t), -1), order="F")
        for line, exact in enumerate([0 * t, 4 + t, 0 * t, 3 * (4 + t) ** 2]):
            mean, samp = m[line, :, 0], m[line, :, 2]
            assert np.all(np.abs(mean - exact) < 5 * samp + 1e-3 * np.max(np.abs(exact) + 1)), line


def test_philox_k_stream_is_its_own_standard_normal_stream():
    """k-space draws (bit 15 of the fourth counter word) differ from the x-space draws of the
    same (site, trajectory, draw, component) and are standard normal."""
    zx = philox.normals(2, 4096, 64, 5, 3, 7, 0, 1)
    zk = philox.normals(2, 4096, 64, 5, 3, 7, 0, 1, kstream=True)
    assert np.mean(zx == zk) < 1e-4  # independent streams: equal values only by coincidence
    assert abs(zk.mean()) < 0.01 and abs(zk.var() - 1) < 0.01
    assert abs(np.corrcoef(zx.ravel(), zk.ravel())[0, 1]) < 0.01
