"""GPU parity of the resident path against the CPU oracle.

Each case runs one or more ensemble blocks through the device p.path
replacement (C ABI xs_run_path) and through the oracle's xpath with the same
Philox noise, and compares the block-mean observables av.  Tolerances:
FP64 fields: 1e-10 relative to the largest |av|; FP32 fields (FP64 tables and
moments): 2e-4 relative.
"""
import numpy as np
import pytest

from oracle import xspde_ref as X
from tests.gpu_util import oracle_block_av, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 2e-4


def _gpu(pdict, blocks, nc, a_in=None, a_out=False, path_kind=0):
    from xspde_matlab_b200 import GpuPath, xpreferences
    p = xpreferences([pdict])[0]
    g = GpuPath(p, path_kind)
    return g.run_path(blocks[0], len(blocks), nc, a_in=a_in, a_out=a_out)


def _compare(pg, po, blocks, ncs, tol):
    for nc in ncs:
        av_g, _ = _gpu(pg, blocks, nc)
        for i, b in enumerate(blocks):
            av_o, _ = oracle_block_av(po, b, nc)
            for o in range(len(av_o)):
                e = rel_err(av_g[i][o].reshape(-1, order="F"), av_o[o].reshape(-1, order="F"))
                assert e < tol, (nc, b, o, e)


SNLS = dict(dimensions=2, points=[11, 64], ranges=[1.0, 10.0], steps=4, ensembles=[8, 2, 1], noises=2)


def _snls(method, checks, precision="fp64", **kw):
    g = dict(SNLS, method=method, checks=checks, precision=precision,
             deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2",
             observe=["@(a,p) a.*conj(a)", "@(a,p) real(a)"], **kw)
    o = dict(SNLS, method=method, checks=checks,
             deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.01 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a), lambda a, p: np.real(a)], **kw)
    return g, o


@pytest.mark.parametrize("method", ["MP", "RK4"])
@pytest.mark.parametrize("checks", [0, 1])
def test_snls_1d_fp64(method, checks):
    g, o = _snls(method, checks)
    _compare(g, o, [0, 1], [1, 2] if checks else [1], FP64_TOL)


def test_snls_1d_fp32_bound():
    g, o = _snls("MP", 1, precision="fp32")
    _compare(g, o, [0, 1], [1, 2], FP32_TOL)


@pytest.mark.parametrize("method", ["Euler", "RK2", "Implicit", "MP", "RK4"])
def test_kubo_sde_methods(method):
    base = dict(dimensions=1, points=[11], ranges=[2.0], steps=5, ensembles=[64, 2, 1], noises=1, method=method,
                checks=1)
    g = dict(base, deriv="@(a,w,p) 1i*w.*a", initial="@(w,p) 1+0*w",
             observe=["@(a,p) real(a(1,:))", "@(a,p) a(1,:).*conj(a(1,:))"])
    o = dict(base, deriv=lambda a, w, p: 1j * w * a, initial=lambda w, p: 1 + 0 * w,
             observe=[lambda a, p: np.real(a[0:1]), lambda a, p: a[0:1] * np.conj(a[0:1])])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_dpo_positive_p_two_fields():
    base = dict(dimensions=1, fields=2, noises=2, points=[6], ranges=[1.0], steps=20, ensembles=[32, 2, 1],
                method="MP", checks=1)
    g = dict(base, params={"gam": 1.0, "eps": 1.3, "chi": 1e-3},
             deriv="@(a,w,p) [-p.gam*a(1,:)+p.eps*a(2,:)-p.chi*a(1,:).^2.*a(2,:)+sqrt(-p.chi*a(1,:).^2).*w(1,:);"
                   " -p.gam*a(2,:)+p.eps*a(1,:)-p.chi*a(2,:).^2.*a(1,:)+sqrt(-p.chi*a(2,:).^2).*w(2,:)]",
             initial="@(v,p) [1+0.5i+0*v(1,:); 1-0.5i+0*v(2,:)]",
             observe=["@(a,p) real(a(1,:).*a(2,:))", "@(a,p) a"])
    gam, eps, chi = 1.0, 1.3, 1e-3

    def deriv(a, w, p):
        a1, a2 = a[0:1], a[1:2]
        return np.concatenate([-gam * a1 + eps * a2 - chi * a1 ** 2 * a2 + np.sqrt(-chi * a1 ** 2 + 0j) * w[0:1],
                               -gam * a2 + eps * a1 - chi * a2 ** 2 * a1 + np.sqrt(-chi * a2 ** 2 + 0j) * w[1:2]])
    o = dict(base, deriv=deriv,
             initial=lambda v, p: np.concatenate([1 + 0.5j + 0 * v[0:1], 1 - 0.5j + 0 * v[1:2]]),
             observe=[lambda a, p: np.real(a[0:1] * a[1:2]), lambda a, p: a])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_gpe_2d_small_periodic():
    base = dict(dimensions=3, points=[6, 16, 12], ranges=[0.5, 8.0, 6.0], steps=3, ensembles=[4, 2, 1], noises=2,
                method="MP", checks=1)
    g = dict(base, deriv="@(a,w,p) (1-abs(a).^2).*a - 0.5i*abs(a).^2.*a + 0.05*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) 1 + 0.1*(v(1,:)+1i*v(2,:))/sqrt(2)", linear="@(p) (1i+0.1)*(p.Dx.^2+p.Dy.^2)",
             observe=["@(a,p) abs(a).^2", "@(a,p) Int(abs(a).^2, p)", "@(a,p) Ave(real(a), p)"])
    o = dict(base, deriv=lambda a, w, p: (1 - abs(a) ** 2) * a - 0.5j * abs(a) ** 2 * a
             + 0.05 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: 1 + 0.1 * (v[0:1] + 1j * v[1:2]) / np.sqrt(2),
             linear=lambda p: (1j + 0.1) * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: X.Int(abs(a) ** 2, p), lambda a, p: X.Ave(np.real(a), p)])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_all_boundary_types_stochastic_heat():
    bnd = [[1, 1], [-1, -1], [1, -1], [-1, 1], [0, 0]]
    base = dict(dimensions=2, fields=5, noises=5, points=[9, 21], ranges=[0.4, np.pi], origins=[0, 0], steps=2,
                ensembles=[4, 2, 1], method="MP", checks=1, boundaries=[None, bnd])
    g = dict(base, deriv="@(a,w,p) 0.1*w - 0.2*a.*conj(a).*a",
             initial="@(v,p) [4*sin(p.x)+sin(2*p.x); 5+4*cos(p.x)+cos(2*p.x); 4*sin(p.x/2)+sin(3*p.x/2);"
                     " 4*cos(p.x/2)+cos(3*p.x/2); 2+cos(2*p.x/1.02)+sin(4*p.x/1.02)]",
             linear="@(p) p.Dx.^2", observe=["@(a,p) a", "@(a,p) Int(abs(a).^2, p.dx, [0 0; 0.5 2.5], p)"])
    x = None

    def init(v, p):
        x = p.x
        return np.concatenate([4 * np.sin(x) + np.sin(2 * x), 5 + 4 * np.cos(x) + np.cos(2 * x),
                               4 * np.sin(x / 2) + np.sin(3 * x / 2), 4 * np.cos(x / 2) + np.cos(3 * x / 2),
                               2 + np.cos(2 * x / 1.02) + np.sin(4 * x / 1.02)], axis=0)
    o = dict(base, deriv=lambda a, w, p: 0.1 * w - 0.2 * a * np.conj(a) * a, initial=init,
             linear=lambda p: p.Dx ** 2,
             observe=[lambda a, p: a, lambda a, p: X.Int(abs(a) ** 2, p.dx, [[0, 0], [0.5, 2.5]], p)])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_a_in_a_out_roundtrip():
    g, o = _snls("RK4", 0)
    av_o, b_o = oracle_block_av(o, 1, 1)
    inp = X.xpreferences([o])[0]
    a0 = np.broadcast_to(np.exp(-inp.x ** 2), inp.ca).astype(complex)
    av_g, a_g = _gpu(g, [1], 1, a_in=a0, a_out=True)
    assert rel_err(a_g, b_o) < FP64_TOL
    assert rel_err(av_g[0][0], av_o[0]) < FP64_TOL


@pytest.mark.parametrize("method", ["MP", "RK4"])
def test_field_in_device_memory_2d_periodic_fp64(method):
    """128 x 128 FP64 (256 KB per array) exceeds shared memory: the resident
    kernel keeps field, scratch and (RK4) noise arrays in per-CTA device-memory
    slices."""
    base = dict(dimensions=3, points=[3, 128, 128], ranges=[0.2, 20.0, 20.0], steps=3, ensembles=[2, 2, 1],
                noises=2, method=method, checks=1)
    g = dict(base, deriv="@(a,w,p) 1i*abs(a).^2.*a + 0.02*(w(1,:)+1i*w(2,:))",
             initial="@(v,p) exp(-(p.x.^2+p.y.^2)/8) + 0.1*v(1,:)", linear="@(p) 0.5i*(p.Dx.^2+p.Dy.^2)",
             observe=["@(a,p) abs(a).^2", "@(a,p) Int(abs(a).^2, p)"])
    o = dict(base, deriv=lambda a, w, p: 1j * abs(a) ** 2 * a + 0.02 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-(p.x ** 2 + p.y ** 2) / 8) + 0.1 * v[0:1],
             linear=lambda p: 0.5j * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: X.Int(abs(a) ** 2, p)])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_field_in_device_memory_3d_dst_dct_fp64():
    """3D lattice with Neumann (DCT-I), Dirichlet (DST-I) and mixed
    Neumann-Dirichlet (DCT-III/II) boundaries, too large for shared memory;
    Allen-Cahn drift with noise."""
    base = dict(dimensions=4, points=[3, 24, 20, 16], ranges=[0.1, 6.0, 5.0, 4.0], steps=2, ensembles=[2, 2, 1],
                noises=1, inrandoms=1, method="MP", checks=1, boundaries=[None, [[-1, -1]], [[1, 1]], [[-1, 1]]])
    g = dict(base, deriv="@(a,w,p) a - a.^3 + 0.1*w(1,:)", initial="@(v,p) 0.3*v(1,:) + 0.5",
             linear="@(p) 0.05*(p.Dx.^2+p.Dy.^2+p.Dz.^2)",
             observe=["@(a,p) abs(a).^2", "@(a,p) Int(real(a).^2, p)"])
    o = dict(base, deriv=lambda a, w, p: a - a ** 3 + 0.1 * w[0:1], initial=lambda v, p: 0.3 * v[0:1] + 0.5,
             linear=lambda p: 0.05 * (p.Dx ** 2 + p.Dy ** 2 + p.Dz ** 2),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: X.Int(np.real(a) ** 2, p)])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_two_fields_a_in_a_out_fp64():
    """Two-component field through the host layout a(fields, ens): initial field
    in, final field and block means out (device-side reordering both ways)."""
    base = dict(dimensions=1, fields=2, noises=2, points=[4], ranges=[0.5], steps=5, ensembles=[16, 1, 1],
                method="MP", checks=0)
    g = dict(base, params={"gam": 1.0, "eps": 1.2, "chi": 1e-3},
             deriv="@(a,w,p) [-p.gam*a(1,:)+p.eps*a(2,:)-p.chi*a(1,:).^2.*a(2,:)+sqrt(-p.chi*a(1,:).^2).*w(1,:);"
                   " -p.gam*a(2,:)+p.eps*a(1,:)-p.chi*a(2,:).^2.*a(1,:)+sqrt(-p.chi*a(2,:).^2).*w(2,:)]",
             initial="@(v,p) [1+0*v(1,:); 1+0*v(2,:)]", observe=["@(a,p) real(a(1,:).*a(2,:))", "@(a,p) a"])
    gam, eps, chi = 1.0, 1.2, 1e-3

    def deriv(a, w, p):
        a1, a2 = a[0:1], a[1:2]
        return np.concatenate([-gam * a1 + eps * a2 - chi * a1 ** 2 * a2 + np.sqrt(-chi * a1 ** 2 + 0j) * w[0:1],
                               -gam * a2 + eps * a1 - chi * a2 ** 2 * a1 + np.sqrt(-chi * a2 ** 2 + 0j) * w[1:2]])
    rng = np.random.default_rng(3)
    a0 = np.asfortranarray(rng.normal(size=(2, 16)) + 1j * rng.normal(size=(2, 16)))
    o = dict(base, deriv=deriv, initial=lambda v, p: a0, observe=[lambda a, p: np.real(a[0:1] * a[1:2]),
                                                                   lambda a, p: a])
    av_o, b_o = oracle_block_av(o, 0, 1)
    av_g, a_g = _gpu(g, [0], 1, a_in=a0, a_out=True)
    assert rel_err(a_g, b_o) < FP64_TOL
    for k in range(2):
        assert rel_err(av_g[0][k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F")) < FP64_TOL


def test_finite_difference_observables_fp64():
    """D1/D2 (Applications/SPDE/D1.m, D2.m) in observables: three components with
    periodic, Neumann and Dirichlet boundaries, site values and an integral."""
    bnd = [[0, 0], [-1, -1], [1, 1]]
    base = dict(dimensions=2, fields=3, noises=3, points=[3, 24], ranges=[0.1, 6.0], steps=2, ensembles=[4, 2, 1],
                method="MP", checks=1, boundaries=[None, bnd])
    g = dict(base, deriv="@(a,w,p) -0.2*a + 0.1*w", initial="@(v,p) [sin(p.x); cos(p.x); sin(p.x/2)] + 0.2*v",
             linear="@(p) 0.3*p.Dx.^2",
             observe=["@(a,p) D1(a,2,p)", "@(a,p) D2(a,p)", "@(a,p) Int(abs(D1(a(2,:),2,p)).^2, p)"])

    def init(v, p):
        return np.concatenate([np.sin(p.x), np.cos(p.x), np.sin(p.x / 2)], axis=0) + 0.2 * v
    o = dict(base, deriv=lambda a, w, p: -0.2 * a + 0.1 * w, initial=init, linear=lambda p: 0.3 * p.Dx ** 2,
             observe=[lambda a, p: X.D1(a, 1, p), lambda a, p: X.D2(a, 1, p),
                      lambda a, p: X.Int(abs(X.D1(a, 1, p)[1:2]) ** 2, p)])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def _bfun(a, c, d, p):
    s, k = np.sin(2 * p.t), np.cos(p.t)
    return [[1 + 0.5 * s, 2 - k], [0.3 * k, -0.2 * s], [0.7 + s, 0.1 * k], [0.2 * s, 1 + 0.3 * k]]


def test_boundary_values_all_types_stochastic_fp64():
    """Time-dependent boundary values (p.boundfun, xpatch.m + xsetbound.m) for
    Dirichlet-Dirichlet, Neumann-Neumann, Dirichlet-Neumann and Neumann-Dirichlet
    components, with noise, merged-step-free MP and both check passes."""
    bnd = [[1, 1], [-1, -1], [1, -1], [-1, 1]]
    base = dict(dimensions=2, fields=4, noises=4, points=[4, 25], ranges=[0.3, 4.0], origins=[0.2, -1.0], steps=3,
                ensembles=[4, 2, 1], method="MP", checks=1, boundaries=[None, bnd], boundfun=_bfun)
    g = dict(base, deriv="@(a,w,p) -0.3*a.*conj(a).*a + 0.05*w", initial="@(v,p) 1 + 0.2*cos(p.x) + 0.1*v",
             linear="@(p) (0.4+0.2i)*p.Dx.^2", observe=["@(a,p) a", "@(a,p) Int(abs(a).^2, p)"])
    o = dict(base, deriv=lambda a, w, p: -0.3 * a * np.conj(a) * a + 0.05 * w,
             initial=lambda v, p: 1 + 0.2 * np.cos(p.x) + 0.1 * v, linear=lambda p: (0.4 + 0.2j) * p.Dx ** 2,
             observe=[lambda a, p: a, lambda a, p: X.Int(abs(a) ** 2, p)])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


@pytest.mark.parametrize("method", ["MP", "RK4"])
def test_time_spectrum_sde_fp64(method):
    """Observables on the time spectrum of the field (p.transforms{n}(1),
    Simulator/xpath.m:46-106) beside a time-domain one; both check passes (the fine
    pass records the mean of its two half steps)."""
    base = dict(dimensions=1, points=[24], ranges=[6.0], steps=3, ensembles=[32, 2, 1], noises=2, method=method,
                checks=1, transforms=[[0], [1], [1]])
    g = dict(base, initial="@(w,p) (w(1,:)+1i*w(2,:))/sqrt(2)", deriv="@(a,w,p) (0.5i-1)*a + w(1,:)+1i*w(2,:)",
             observe=["@(a,p) a.*conj(a)", "@(a,p) a.*conj(a)", "@(a,p) a"])
    o = dict(base, initial=lambda w, p: (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             deriv=lambda a, w, p: (0.5j - 1) * a + w[0:1] + 1j * w[1:2],
             observe=[lambda a, p: a * np.conj(a), lambda a, p: a * np.conj(a), lambda a, p: a])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_time_spectrum_sde_fp32_bound():
    base = dict(dimensions=1, points=[24], ranges=[6.0], steps=3, ensembles=[32, 2, 1], noises=2, method="MP",
                checks=1, transforms=[[0], [1]])
    g = dict(base, precision="fp32", initial="@(w,p) (w(1,:)+1i*w(2,:))/sqrt(2)",
             deriv="@(a,w,p) -a + w(1,:)+1i*w(2,:)", observe=["@(a,p) a.*conj(a)", "@(a,p) a.*conj(a)"])
    o = dict(base, initial=lambda w, p: (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             deriv=lambda a, w, p: -a + w[0:1] + 1j * w[1:2],
             observe=[lambda a, p: a * np.conj(a), lambda a, p: a * np.conj(a)])
    _compare(g, o, [0, 1], [1, 2], FP32_TOL)


def test_time_spectrum_pde_kspace_integral_fp64():
    """Time spectrum of a 1D stochastic NLS field: the (w, x) spectrum, the (w, k)
    spectrum (time and space transforms together) and the integral of the (w, x)
    spectrum."""
    base = dict(dimensions=2, points=[10, 32], ranges=[2.0, 10.0], steps=3, ensembles=[4, 2, 1], noises=2,
                method="MP", checks=1, transforms=[[0, 0], [1, 0], [1, 1], [1, 0]])
    g = dict(base, deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.1*(w(1,:)+1i*w(2,:))", initial="@(v,p) exp(-p.x.^2)",
             linear="@(p) 1i*p.Dx.^2",
             observe=["@(a,p) a.*conj(a)", "@(a,p) a.*conj(a)", "@(a,p) a.*conj(a)", "@(a,p) Int(a.*conj(a),p)"])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.1 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a)] * 3 + [lambda a, p: X.Int(a * np.conj(a), p)])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_time_spectrum_field_in_device_memory_fp64():
    """128 x 128 FP64 lattice (field in per-CTA device-memory slices) with a
    time-spectrum observable."""
    base = dict(dimensions=3, points=[4, 128, 128], ranges=[0.3, 20.0, 20.0], steps=2, ensembles=[2, 1, 1],
                noises=2, method="MP", checks=1, transforms=[[0, 0, 0], [1, 0, 0]])
    g = dict(base, deriv="@(a,w,p) 1i*abs(a).^2.*a + 0.02*(w(1,:)+1i*w(2,:))",
             initial="@(v,p) exp(-(p.x.^2+p.y.^2)/8)", linear="@(p) 0.5i*(p.Dx.^2+p.Dy.^2)",
             observe=["@(a,p) abs(a).^2", "@(a,p) abs(a).^2"])
    o = dict(base, deriv=lambda a, w, p: 1j * abs(a) ** 2 * a + 0.02 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-(p.x ** 2 + p.y ** 2) / 8),
             linear=lambda p: 0.5j * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: abs(a) ** 2])
    _compare(g, o, [0], [1, 2], FP64_TOL)


@pytest.mark.parametrize("nc", [1, 2])
def test_raw_trajectories_two_fields_fp64(nc):
    """p.rawdata (Simulator/xpath.m:73-78): the field of every trajectory at every
    output time, [fields, points(1), space, ens], for two blocks in one call."""
    from xspde_matlab_b200 import GpuPath, xpreferences
    base = dict(dimensions=2, fields=2, noises=2, points=[6, 16], ranges=[0.6, 6.0], steps=2, ensembles=[4, 2, 1],
                method="MP", checks=1, rawdata=1)
    g = dict(base, deriv="@(a,w,p) [1i*a(2,:) + 0.1*w(1,:); 1i*a(1,:) - 0.2*a(2,:) + 0.1*w(2,:)]",
             initial="@(v,p) [exp(-p.x.^2); 0.5 + 0.1*v(1,:)]", linear="@(p) 0.2i*p.Dx.^2",
             observe=["@(a,p) a(1,:).*conj(a(2,:))"])
    o = dict(base, deriv=lambda a, w, p: np.concatenate([1j * a[1:2] + 0.1 * w[0:1],
                                                         1j * a[0:1] - 0.2 * a[1:2] + 0.1 * w[1:2]]),
             initial=lambda v, p: np.concatenate([np.exp(-p.x ** 2) + 0 * v[0:1], 0.5 + 0.1 * v[0:1]]),
             linear=lambda p: 0.2j * p.Dx ** 2, observe=[lambda a, p: a[0:1] * np.conj(a[1:2])])
    path = GpuPath(xpreferences([g])[0])
    av, _, raw = path.run_path(0, 2, nc, raw=True)
    assert raw.shape == (2, 6, 16, 8)
    for b in range(2):
        av_o, b_o, raw_o = oracle_block_av(o, b, nc)
        assert rel_err(raw[..., 4 * b:4 * b + 4], raw_o) < FP64_TOL
        assert rel_err(av[b][0].reshape(-1, order="F"), av_o[0].reshape(-1, order="F")) < FP64_TOL


def _planar_init(u, v, p):
    return np.concatenate([(u[0:1] + 1j * u[1:2]) / np.sqrt(2), (v[0:1] + 1j * v[1:2]) / np.sqrt(2)], axis=0)


def _planar_deriv(a, w, z, p):
    return np.concatenate([(w[0:1] + 1j * w[1:2]) / np.sqrt(2) - 0.1 * a[0:1] * z[0:1],
                           (z[0:1] + 1j * z[1:2]) / np.sqrt(2)], axis=0)


@pytest.mark.parametrize("method", ["MP", "RK4"])
def test_knoise_planar_two_cells_fp64(method):
    """x-space and k-filtered noises and randoms together (Examples/SPDE_3D/Planar.m
    with a multiplicative k-noise term): deriv(a, w, z, p), initial(u, v, p), both
    check passes, 16 x 12 lattice (FFT and dense DFT dimensions)."""
    base = dict(dimensions=3, fields=2, ranges=[0.4, 5, 5], points=[5, 16, 12], steps=2, noises=2, knoises=2,
                inrandoms=2, krandoms=2, ensembles=[3, 2, 1], method=method, checks=1)
    g = dict(base, initial="@(u,v,p) [(u(1,:)+1i*u(2,:))/sqrt(2); (v(1,:)+1i*v(2,:))/sqrt(2)]",
             deriv="@(a,w,z,p) [(w(1,:)+1i*w(2,:))/sqrt(2) - 0.1*a(1,:).*z(1,:); (z(1,:)+1i*z(2,:))/sqrt(2)]",
             linear="@(p) 0.5i*(p.Dx.^2+p.Dy.^2)",
             observe=["@(a,p) a(1,:).*conj(a(1,:))", "@(a,p) Int(a(2,:).*conj(a(2,:)),p)", "@(a,p) a(2,:)"])
    o = dict(base, initial=_planar_init, deriv=_planar_deriv, linear=lambda p: 0.5j * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: a[0:1] * np.conj(a[0:1]), lambda a, p: X.Int(a[1:2] * np.conj(a[1:2]), p),
                      lambda a, p: a[1:2]])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def _gpe_filter(v, p):
    return v * np.exp(-p.kx ** 2 - p.ky ** 2)


@pytest.mark.parametrize("points,precision,tol", [([4, 20, 20], "fp64", FP64_TOL), ([4, 16, 16], "fp64", FP64_TOL),
                                                  ([4, 16, 16], "fp32", FP32_TOL)])
def test_knoise_filtered_gpe(points, precision, tol):
    """Examples/SPDE_3D/GPE.m form: only k-filtered noises and randoms, both filtered
    by exp(-kx^2 - ky^2) (p.nfilter, p.rfilter), so the drift's noise argument is the
    k-noise cell: deriv(a, w, p) with w = z."""
    base = dict(dimensions=3, points=points, ranges=[0.3, 20, 20], knoises=2, krandoms=2, ensembles=[2, 2, 1],
                method="MP", checks=1, nfilter=_gpe_filter, rfilter=_gpe_filter)
    g = dict(base, precision=precision,
             initial="@(w,p) (p.x+1i*p.y)./(1+10*(p.x.^2+p.y.^2)) + 0.1*(w(1,:)+1i*w(2,:))",
             deriv="@(a,w,p) -1i*a.*(0.01*(p.x.^2+p.y.^2) + conj(a).*a) + 0.1*(w(1,:)+1i*w(2,:))",
             linear="@(p) 0.5i*(p.Dx.^2+p.Dy.^2)", observe=["@(a,p) a.*conj(a)", "@(a,p) Int(abs(a).^2,p)"])
    o = dict(base, initial=lambda w, p: (p.x + 1j * p.y) / (1 + 10 * (p.x ** 2 + p.y ** 2)) + 0.1 * (w[0:1] + 1j * w[1:2]),
             deriv=lambda a, w, p: -1j * a * (0.01 * (p.x ** 2 + p.y ** 2) + np.conj(a) * a) + 0.1 * (w[0:1] + 1j * w[1:2]),
             linear=lambda p: 0.5j * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: a * np.conj(a), lambda a, p: X.Int(abs(a) ** 2, p)])
    _compare(g, o, [0, 1], [1, 2], tol)


def test_knoise_field_in_device_memory_rk4_fp64():
    """128 x 128 lattice (field, scratch and k-noise arrays in device memory), RK4."""
    base = dict(dimensions=3, points=[3, 128, 128], ranges=[0.1, 20, 20], knoises=2, krandoms=2, ensembles=[2, 1, 1],
                method="RK4", checks=1, nfilter=_gpe_filter, rfilter=_gpe_filter)
    g = dict(base, initial="@(w,p) exp(-(p.x.^2+p.y.^2)/8) + 0.1*(w(1,:)+1i*w(2,:))",
             deriv="@(a,w,p) -1i*a.*conj(a).*a + 0.1*(w(1,:)+1i*w(2,:))", linear="@(p) 0.5i*(p.Dx.^2+p.Dy.^2)",
             observe=["@(a,p) a.*conj(a)"])
    o = dict(base, initial=lambda w, p: np.exp(-(p.x ** 2 + p.y ** 2) / 8) + 0.1 * (w[0:1] + 1j * w[1:2]),
             deriv=lambda a, w, p: -1j * a * np.conj(a) * a + 0.1 * (w[0:1] + 1j * w[1:2]),
             linear=lambda p: 0.5j * (p.Dx ** 2 + p.Dy ** 2), observe=[lambda a, p: a * np.conj(a)])
    _compare(g, o, [0], [1, 2], FP64_TOL)


def test_block_means_are_compensated_sums_fp64():
    """Block means sum the trajectories with Neumaier compensation: the values
    [1e16, 1, -1e16, 1] average to exactly 0.5 (a plain left-to-right FP64 sum
    loses both ones against 1e16 and gives 0.25)."""
    base = dict(dimensions=1, points=[2], ranges=[0.1], steps=1, ensembles=[4, 1, 1], noises=1, method="MP",
                checks=0)
    g = dict(base, deriv="@(a,w,p) 0*a", initial="@(v,p) 0", observe=["@(a,p) real(a)"])
    a0 = np.array([[1e16, 1.0, -1e16, 1.0]], dtype=complex)
    av, _ = _gpu(g, [0], 1, a_in=a0)
    assert np.all(np.real(av[0][0]) == 0.5), av[0][0]


def _a1(w):
    return (w[0:1] + 1j * w[1:2]) / 2


@pytest.mark.parametrize("method", ["MP", "RK4"])
def test_auxiliary_fields_with_spectra_fp64(method):
    """Auxiliary fields (p.auxfields, p.define; xpath.m:36-45, xensemble.m:74-77):
    Examples/SDE_1D/Quantum.m form, input and output fields defined from the
    oscillator and its noise, observed in time and as time spectra, both check passes."""
    base = dict(points=[41], ranges=[8.0], auxfields=2, noises=2, ensembles=[16, 2, 1], method=method, checks=1,
                transforms=[[1], [1], [1], [0]])
    g = dict(base, initial="@(w,p) (w(1,:)+1i*w(2,:))/2", deriv="@(a,w,p) -a(1,:)+sqrt(2)*(w(1,:)+1i*w(2,:))/2",
             define="@(a,w,p) [(w(1,:)+1i*w(2,:))/2; sqrt(2)*a(1,:)-(w(1,:)+1i*w(2,:))/2]",
             observe=["@(a,x,p) abs(a(1,:)).^2", "@(a,x,p) abs(x(1,:)).^2", "@(a,x,p) abs(x(2,:)).^2",
                      "@(a,x,p) x(2,:)"])
    o = dict(base, initial=lambda w, p: _a1(w), deriv=lambda a, w, p: -a[0:1] + np.sqrt(2) * _a1(w),
             define=lambda a, w, p: np.concatenate([_a1(w), np.sqrt(2) * a[0:1] - _a1(w)]),
             observe=[lambda a, x, p: abs(a[0:1]) ** 2, lambda a, x, p: abs(x[0:1]) ** 2,
                      lambda a, x, p: abs(x[1:2]) ** 2, lambda a, x, p: x[1:2]])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_auxiliary_field_time_dependent_define_fp64():
    """Examples/SDE_1D/Kubodefine.m form: define = exp(5i t) a reads p.t, which
    stays at the start of the step for both evaluations around the method."""
    base = dict(points=[21], ranges=[4.0], auxfields=1, noises=1, ensembles=[32, 2, 1], method="RK4", checks=1,
                transforms=[[0], [1], [1]])
    g = dict(base, initial="@(w,p) 1+0*w", deriv="@(a,w,p) 1i*w.*a", define="@(a,w,p) exp(5*1i*p.t).*a",
             observe=["@(a,x,p) a", "@(a,x,p) a.*conj(a)", "@(a,x,p) x.*conj(x)"])
    o = dict(base, initial=lambda w, p: 1 + 0 * w, deriv=lambda a, w, p: 1j * w * a,
             define=lambda a, w, p: np.exp(5j * p.t) * a,
             observe=[lambda a, x, p: a, lambda a, x, p: a * np.conj(a), lambda a, x, p: x * np.conj(x)])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_auxiliary_field_on_a_lattice_fp64():
    """An auxiliary field on a 1D lattice with noise in its definition, observed
    per site and through an integral."""
    base = dict(dimensions=2, points=[6, 32], ranges=[0.5, 8.0], auxfields=1, noises=2, ensembles=[4, 2, 1],
                method="MP", checks=1)
    g = dict(base, deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.1*(w(1,:)+1i*w(2,:))", initial="@(v,p) exp(-p.x.^2)",
             linear="@(p) 1i*p.Dx.^2", define="@(a,w,p) a.*conj(a) + w(1,:)",
             observe=["@(a,x,p) a.*conj(a)", "@(a,x,p) Int(real(x),p)", "@(a,x,p) x"])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.1 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
             define=lambda a, w, p: a * np.conj(a) + w[0:1],
             observe=[lambda a, x, p: a * np.conj(a), lambda a, x, p: X.Int(np.real(x), p), lambda a, x, p: x])
    _compare(g, o, [0, 1], [1, 2], FP64_TOL)


def test_auxiliary_field_on_a_device_memory_lattice_fp64():
    """An auxiliary cell on a 128 x 128 lattice (field, scratch, auxiliary chunks and
    the spectrum record in device memory), observed in time and as a spectrum."""
    base = dict(dimensions=3, points=[4, 128, 128], ranges=[0.3, 20.0, 20.0], steps=2, ensembles=[2, 1, 1],
                noises=2, auxfields=1, method="MP", checks=1, transforms=[[0, 0, 0], [1, 0, 0]])
    g = dict(base, deriv="@(a,w,p) 1i*abs(a).^2.*a + 0.02*(w(1,:)+1i*w(2,:))",
             initial="@(v,p) exp(-(p.x.^2+p.y.^2)/8)", linear="@(p) 0.5i*(p.Dx.^2+p.Dy.^2)",
             define="@(a,w,p) abs(a).^2 + 0.1*w(2,:)", observe=["@(a,x,p) Int(real(x),p)", "@(a,x,p) abs(x).^2"])
    o = dict(base, deriv=lambda a, w, p: 1j * abs(a) ** 2 * a + 0.02 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-(p.x ** 2 + p.y ** 2) / 8),
             linear=lambda p: 0.5j * (p.Dx ** 2 + p.Dy ** 2), define=lambda a, w, p: abs(a) ** 2 + 0.1 * w[1:2],
             observe=[lambda a, x, p: X.Int(np.real(x), p), lambda a, x, p: abs(x) ** 2])
    _compare(g, o, [0], [1, 2], FP64_TOL)


def test_noise_argument_without_noise_cells_is_zero_fp64():
    """With noises = 0 the drift's w is the scalar 0, as xnoise.m passes it."""
    base = dict(dimensions=2, points=[5, 32], ranges=[0.5, 8.0], steps=2, ensembles=[4, 1, 1], noises=0,
                inrandoms=0, method="RK4", checks=1)
    g = dict(base, deriv="@(a,w,p) 1i*abs(a).^2.*a + 3*w", initial="@(v,p) exp(-p.x.^2) + v",
             linear="@(p) 1i*p.Dx.^2", observe=["@(a,p) abs(a).^2"])
    o = dict(base, deriv=lambda a, w, p: 1j * abs(a) ** 2 * a + 3 * w, initial=lambda v, p: np.exp(-p.x ** 2) + v,
             linear=lambda p: 1j * p.Dx ** 2, observe=[lambda a, p: abs(a) ** 2])
    _compare(g, o, [0], [1, 2], FP64_TOL)
