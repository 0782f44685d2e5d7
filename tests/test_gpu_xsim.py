"""End to end through the host mirror of xsim (xspde_matlab_b200.xsim) with
the device path: the reference's own deterministic golden errors
(Examples/Batchtest.m:67-75, accepted within a factor 1.001 at :81) and the
full error/data output of a stochastic run against the oracle's xsim."""
import warnings

import numpy as np
import pytest

from oracle import xspde_ref as X

pytestmark = pytest.mark.gpu


def sech(x):
    return 1 / np.cosh(x)


GOLDEN = {
    # Examples/SPDE_2D/Soliton.m
    "Soliton": dict(dimensions=2, checks=0, order=2, initial="@(v,p) sech(p.x)",
                    deriv="@(a,~,~) 1i*a.*(conj(a).*a)", linear="@(p) 0.5*1i*(p.Dx.^2-1.0)",
                    compare=lambda p: sech(p.x)),
    # Examples/SPDE_2D/Characteristic.m
    "Characteristic": dict(dimensions=2, initial="@(w,p) sech(2.*(p.x+2.5))", linear="@(p) -p.Dx",
                           points=[51, 35], observe=["@(a,~) a", "@(a,~) a.^2"], axes=[None, [0, 18]],
                           compare=[None, lambda p: sech(2 * (p.t - 2.5)) ** 2]),
    # Examples/SPDE_2D/SolitonAv.m
    "SolitonAv": dict(dimensions=2, observe=["@(a,p) Ave(real(a),p.dx,p)", "@(a,p) Int(real(a),p.dx,p)"],
                      initial="@(v,p) sech(p.x)", deriv="@(a,~,~) 1i*a.*(conj(a).*a)",
                      linear="@(p) 0.5*1i*(p.Dx.^2-1.0)",
                      compare=[lambda p: np.pi / 10 + 0 * p.t, lambda p: np.pi + 0 * p.t]),
    # Examples/SPDE_2D/GaussianAv2D.m: k-space observable (p.transforms)
    "GaussianAv2D": dict(dimensions=3, initial="@(v,p) exp(-0.5*(p.x.^2+p.y.^2))", deriv="@(a,w,p) 0*a",
                         observe=["@(a,p) a.*conj(a)", "@(a,p) Ave(a.*conj(a), p.dx, p)",
                                  "@(a,p) Int(a.*conj(a), p.dx, p)", "@(a,p) a.*conj(a)"],
                         linear="@(p) 1i*0.05*(p.Dx.^2+p.Dy.^2)", transforms=[0, 0, 0, [0, 1, 1]],
                         compare=[lambda p: (1 + (p.t / 10) ** 2) ** -1
                                  * np.exp(-(p.x ** 2 + p.y ** 2) / (1 + (p.t / 10) ** 2)), None, None,
                                  lambda r: 1], axes=[None, None, None, [0, -1, -1]]),
    # Examples/SPDE_2D/GaussianKinetic.m: k-space observables with p.kx, p.ky and p.dk integrals
    "GaussianKinetic": dict(dimensions=3, fields=1, ranges=[5, 200, 6], points=[49, 70, 34],
                            initial="@(v,p) sqrt(exp(-p.x.^2/3.3^2 - p.y.^2/0.235^2)/(pi*3.3*0.235))",
                            linear="@(p) 1i*(p.Dx.^2)",
                            observe=["@(a,p) abs(a).^2", "@(a,p) abs(a).^2",
                                     "@(a,p) Int(abs(a).^2.*(p.kx.^2+p.ky.^2), p.dk, p)",
                                     "@(a,p) sqrt(Int(p.y.^2.*abs(a).^2, p.dx, p)./Int(abs(a).^2, p.dx, p))",
                                     "@(a,p) sqrt(Int(p.x.^2.*abs(a).^2, p.dx, p)./Int(abs(a).^2, p.dx, p))",
                                     "@(a,p) sqrt(Int(p.ky.^2.*abs(a).^2, p.dk, p)./Int(abs(a).^2, p.dk, p))"],
                            transforms=[0, [0, 1, 1], [0, 1, 1], 0, 0, [0, 1, 1]],
                            compare=[None, None, lambda p: 1 / (2 * 3.3 ** 2) + 1 / (2 * 0.235 ** 2),
                                     lambda p: 0.235 / np.sqrt(2), None, lambda p: 1 / (np.sqrt(2) * 0.235)]),
    # Examples/SPDE_2D/SolitonDerivN.m: RK4, Neumann (DCT-I) boundaries, D1 finite differences in an observable
    "SolitonDerivN": dict(dimensions=2, points=[101, 101], method="RK4", order=4, ranges=[10, 15],
                          initial="@(v,p) sech(p.x)",
                          observe=["@(a,p) a.*conj(a)", "@(a,p) Int(abs(D1(a,2,p)).^2,p)"],
                          boundaries=[None, [-1, -1]], deriv="@(a,w,p) 1i*a.*(conj(a).*a)",
                          linear="@(p) 0.5i*(p.Dx.^2-1)"),
    # Examples/SPDE_nD/Gaussian3D.m: 35^3 FP64 lattice, beyond shared memory (field in device memory)
    "Gaussian3D": dict(noises=0, dimensions=4, initial="@(w,p) exp(-(p.x.^2+p.y.^2+p.z.^2)/2)",
                       observe=["@(a,p) a.*conj(a)"], linear="@(p) -0.5 + 1i*0.05*(p.Dx.^2+p.Dy.^2+p.Dz.^2)",
                       compare=[lambda p: (1 + (p.t / 10) ** 2) ** -1.5
                                * np.exp(-p.t - (p.x ** 2 + p.y ** 2 + p.z ** 2) / (1 + (p.t / 10) ** 2))]),
}


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_gpu_xsim_batchtest_golden(name, golden_expected):
    from xspde_matlab_b200 import xsim
    e, data, inp = xsim(GOLDEN[name])
    exp = golden_expected[name]
    assert exp / 1.001 < e[0] < exp * 1.001, (name, e[0], exp)


def test_gpu_xsim_stochastic_matches_oracle():
    from xspde_matlab_b200 import xsim
    base = dict(dimensions=2, points=[9, 32], ranges=[1.0, 8.0], steps=3, ensembles=[16, 4, 2], noises=2,
                method="MP", checks=1, order=1)
    g = dict(base, deriv="@(a,w,p) 1i*a.*conj(a).*a - 0.1*a + 0.05*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) exp(-p.x.^2) + 0.01*v(1,:)", linear="@(p) 1i*p.Dx.^2",
             observe=["@(a,p) a.*conj(a)", "@(a,p) Int(abs(a).^2, p)"],
             compare=[None, lambda p: np.sqrt(np.pi / 2) * np.exp(-0.2 * p.t)])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a - 0.1 * a + 0.05 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: np.exp(-p.x ** 2) + 0.01 * v[0:1], linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a), lambda a, p: X.Int(abs(a) ** 2, p)],
             compare=[None, lambda p: np.sqrt(np.pi / 2) * np.exp(-0.2 * p.t)])
    eg, dg, _ = xsim(g)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        eo, do, _ = X.xsim(o)
    keep = [i for i in range(len(eo)) if i != 5]  # error(sx+2) with sx = 3 is the run time
    assert np.allclose(eg[keep], eo[keep], rtol=1e-9, atol=1e-14), (eg, eo)
    for a, b in zip(dg[0], do[0]):
        assert np.allclose(a, b, rtol=1e-9, atol=1e-13)
