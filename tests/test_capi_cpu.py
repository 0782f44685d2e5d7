"""CPU-only checks of the C ABI library: it loads, exports every declared
symbol, reports errors, and NVRTC compiles problem kernels for sm_100a
(compilation needs no GPU)."""
import ctypes
import os
import re

import pytest

from xspde_matlab_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_header_exports_match():
    hdr = open(os.path.join(ROOT, "include", "xspde_b200.h")).read()
    declared = set(re.findall(r"XS_API\s+[\w\s\*]+?\b(xs_\w+)\s*\(", hdr))
    assert declared == set(_lib.EXPORTS)
    L = _lib.lib()
    for name in declared:
        assert hasattr(L, name), name


def test_version_and_error_buffer():
    L = _lib.lib()
    assert b"sm_100a" in L.xs_version()
    h = ctypes.c_void_p()
    assert L.xs_create(None, ctypes.byref(h)) == -7
    assert "null problem" in _lib.last_error()


def _problem(**kw):
    from tests.capi_problems import make_problem
    return make_problem(**kw)


def test_compile_check_cfg1(tmp_path, monkeypatch):
    monkeypatch.setenv("XSPDE_B200_CACHE", str(tmp_path))
    p, keep = _problem()
    log = ctypes.create_string_buffer(1 << 16)
    rc = _lib.lib().xs_compile_check(ctypes.byref(p), log, len(log))
    assert rc == 0, _lib.last_error()
    assert any(f.endswith(".cubin") for f in os.listdir(tmp_path))


@pytest.mark.parametrize("deriv,frag", [
    ("@(a,w,p) D2(b,2,p)", "D2 on the device takes the field a"),
    ("@(a,w,p) a.*q", "unknown identifier 'q'"),
    ("@(a,w,p) a + p.gamma", "unknown parameter 'p.gamma'"),
    ("@(a,w,p) a(3,:)", "out of range"),
    ("@(a,w,p) a + 'x'", "strings"),
])
def test_grammar_rejections(deriv, frag, tmp_path, monkeypatch):
    monkeypatch.setenv("XSPDE_B200_CACHE", str(tmp_path))
    p, keep = _problem(deriv=deriv)
    rc = _lib.lib().xs_compile_check(ctypes.byref(p), None, 0)
    assert rc == -2
    assert frag in _lib.last_error()


def test_named_scalars_and_precision(tmp_path, monkeypatch):
    monkeypatch.setenv("XSPDE_B200_CACHE", str(tmp_path))
    p, keep = _problem(deriv="@(a,w,p) -p.gamma*a + p.eps*conj(a) + sqrt(-p.chi*a.^2).*w(1,:)", precision=1,
                       params={"gamma": 1.0, "eps": 0.5, "chi": 1e-3}, noises=1, dimensions=1, linear="",
                       initial="@(v,p) 1", observe=("@(a,p) a",))
    rc = _lib.lib().xs_compile_check(ctypes.byref(p), None, 0)
    assert rc == 0, _lib.last_error()


def test_kfilter_table_layout_and_pointwise_check():
    """p.nfilter becomes a [components][space] complex table on the FFT-ordered k
    lattice (site index column-major); a filter that is not w .* f(k) is refused."""
    import numpy as np
    from xspde_matlab_b200 import xpreferences
    from xspde_matlab_b200.xsim import _filter_table
    p = xpreferences([dict(dimensions=3, points=[3, 6, 4], ranges=[1.0, 6.0, 4.0], knoises=2)])[0]
    assert p.noises == 0 and p.knoises == 2 and p.inrandoms == 0
    tab = _filter_table(lambda v, p: v * (1 + p.kx ** 2 + 2j * p.ky), 2, p).view(complex).reshape(2, 24)
    kx = 2 * np.pi * np.fft.fftfreq(6, d=6.0 / 5)
    ky = 2 * np.pi * np.fft.fftfreq(4, d=4.0 / 3)
    want = (1 + kx[:, None] ** 2 + 2j * ky[None, :]).reshape(-1, order="F")
    assert np.allclose(tab[0], want) and np.allclose(tab[1], want)
    with pytest.raises(ValueError):
        _filter_table(lambda v, p: v ** 2, 1, p)


def test_knoise_rejections(tmp_path, monkeypatch):
    monkeypatch.setenv("XSPDE_B200_CACHE", str(tmp_path))
    p, keep = _problem(deriv="@(a,z,p) a + z(1,:)", noises=0)
    p.knoises = 1
    rc = _lib.lib().xs_compile_check(ctypes.byref(p), None, 0)
    assert rc == 0, _lib.last_error()
    p.knoises = 40
    assert _lib.lib().xs_compile_check(ctypes.byref(p), None, 0) == -1


def test_absent_noise_and_random_arguments_are_zero(tmp_path, monkeypatch):
    """Without noise or random cells the reference passes the scalar 0 for w and v
    (xnoise.m and xrandom.m start from w{1} = 0), so '0*w' and '1 + v' compile."""
    monkeypatch.setenv("XSPDE_B200_CACHE", str(tmp_path))
    p, keep = _problem(deriv="@(a,w,p) -a + 0.1*w", initial="@(v,p) 1 + v", noises=0, inrandoms=0)
    rc = _lib.lib().xs_compile_check(ctypes.byref(p), None, 0)
    assert rc == 0, _lib.last_error()
    p, keep = _problem(deriv="@(a,w,p) -a + w(2,:)", noises=0)
    assert _lib.lib().xs_compile_check(ctypes.byref(p), None, 0) == -2


def test_zeros_with_literal_sizes(tmp_path, monkeypatch):
    """zeros(n,1,1) / ones(n,1) give n components (Examples/SPDE_2D/Peregrine.m broadcasts its
    initial value to four components this way); other shapes are refused."""
    monkeypatch.setenv("XSPDE_B200_CACHE", str(tmp_path))
    p, keep = _problem(fields=4, noises=0, initial="@(v,p) exp(-p.x.^2) + zeros(4,1,1)", deriv="@(a,w,p) -a + ones(4,1)",
                       observe=("@(a,p) a(4,:)",), linear="")
    rc = _lib.lib().xs_compile_check(ctypes.byref(p), None, 0)
    assert rc == 0, _lib.last_error()
    p, keep = _problem(initial="@(v,p) zeros(2,3)")
    assert _lib.lib().xs_compile_check(ctypes.byref(p), None, 0) == -2


# a 64 x 64 periodic lattice, which the streaming path takes unless a feature rules it out
_LATTICE2D = dict(dimensions=3, points=(5, 64, 64), ranges=(0.5, 10.0, 10.0), ensembles=(8, 2, 1),
                  linear="@(p) 1i*(p.Dx.^2+p.Dy.^2)")


def _flags(vals):
    arr = (ctypes.c_int * len(vals))(*vals)
    return arr


@pytest.mark.parametrize("setup,code,frag", [
    (lambda p: setattr(p, "auxfields", 17), -1, "auxfields must be 0..16"),
    (lambda p: setattr(p, "auxfields", 1), -7, "auxfields given without p.define"),
    (lambda p: (setattr(p, "knoises", 1), setattr(p, "path_kind", 2)), -9, "k-filtered noises are not streamed"),
    (lambda p: (setattr(p, "auxfields", 1), setattr(p, "define", b"@(a,w,p) a"), setattr(p, "path_kind", 2)), -9,
     "auxiliary fields (p.define) are not streamed"),
    (lambda p: (setattr(p, "auxfields", 2), setattr(p, "define", b"@(a,w,p) [a; a; a]")), -1,
     "p.define returns 3 components"),
])
def test_feature_rejections(setup, code, frag, tmp_path, monkeypatch):
    """Argument checks and refusals of the auxiliary-field and k-noise options (C ABI errors, no GPU)."""
    monkeypatch.setenv("XSPDE_B200_CACHE", str(tmp_path))
    p, keep = _problem(**_LATTICE2D)
    setup(p)
    rc = _lib.lib().xs_compile_check(ctypes.byref(p), None, 0)
    assert rc == code, (rc, _lib.last_error())
    assert frag in _lib.last_error()


def test_time_spectrum_refused_on_streaming_path(tmp_path, monkeypatch):
    monkeypatch.setenv("XSPDE_B200_CACHE", str(tmp_path))
    p, keep = _problem(observe=("@(a,p) a.*conj(a)",), **_LATTICE2D)
    flags = _flags([1, 0, 0, 0])
    p.transforms = flags
    p.path_kind = 2
    rc = _lib.lib().xs_compile_check(ctypes.byref(p), None, 0)
    assert rc == -9 and "time-spectrum observables" in _lib.last_error()
    p.path_kind = 1
    assert _lib.lib().xs_compile_check(ctypes.byref(p), None, 0) == 0, _lib.last_error()


def test_partial_int_observable_shape():
    """An Int over x of a 2D lattice is the lattice with x of size 1 in av{o}
    (Applications/SPDE/Int.m:48-70); a nonlinear function of such an Int is refused."""
    import ctypes

    from xspde_matlab_b200 import _lib, xpreferences
    from xspde_matlab_b200.xsim import make_problem
    base = dict(dimensions=3, points=[3, 8, 6], ranges=[1.0, 4.0, 3.0], deriv="@(a,w,p) 0*a",
                initial="@(v,p) 1 + 0*p.x")
    L = _lib.lib()
    p = xpreferences([dict(base, observe=["@(a,p) Int(abs(a).^2, [0, 0.5, 0], p)", "@(a,p) a"])])[0]
    pr, keep = make_problem(p)
    h = ctypes.c_void_p()
    _lib.check(L.xs_create(ctypes.byref(pr), ctypes.byref(h)))
    try:
        dims = (ctypes.c_int * 3)()
        _lib.check(L.xs_observe_shape(h, 0, dims))
        assert list(dims) == [1, 6, 1]
        _lib.check(L.xs_observe_shape(h, 1, dims))
        assert list(dims) == [8, 6, 1]
        assert L.xs_av_doubles_per_block(h) == 2 * 3 * (6 + 48)
    finally:
        L.xs_destroy(h)
    p = xpreferences([dict(base, observe=["@(a,p) Int(abs(a).^2, [0, 0.5, 0], p).^2"])])[0]
    pr, keep = make_problem(p)
    assert L.xs_create(ctypes.byref(pr), ctypes.byref(h)) != 0
    assert "whole observable" in _lib.last_error()
