"""Int/Ave over a subset of the space dimensions (Applications/SPDE/Int.m:48-70,
Ave.m) as the whole observable: the device evaluates the integrand per site and
the host sums the block means over the reduced dimensions (the sum is linear,
so it commutes with the ensemble mean).  Checked against the oracle's block
means in FP64 (1e-10) on a 2D stochastic lattice: Int over x, Int over y with
bounds, Ave over x, and through the host xsim against the oracle's xsim."""
import warnings

import numpy as np
import pytest

from oracle import xspde_ref as X
from tests.gpu_util import oracle_block_av, rel_err

pytestmark = pytest.mark.gpu


def _inputs():
    dx, dy = 8.0 / 15, 6.0 / 11
    base = dict(dimensions=3, points=[4, 16, 12], ranges=[0.5, 8.0, 6.0], steps=2, ensembles=[3, 2, 1], noises=2,
                method="MP", checks=1, precision="fp64")
    g = dict(base, deriv="@(a,w,p) 1i*a.*conj(a).*a - 0.1*a + 0.05*(w(1,:)+1i*w(2,:))",
             initial="@(v,p) exp(-p.x.^2 - 0.5*p.y.^2) + 0.01*v(1,:)", linear="@(p) 1i*(p.Dx.^2 + p.Dy.^2)",
             observe=["@(a,p) Int(abs(a).^2, [0, %r, 0], p)" % dx,
                      "@(a,p) Int(real(a), [0, 0, %r], [0, 0; 0, 0; -1.5, 2.0], p)" % dy,
                      "@(a,p) Ave(a.*conj(a), [0, 1, 0], p)",
                      "@(a,p) abs(a).^2"])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a - 0.1 * a + 0.05 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-p.x ** 2 - 0.5 * p.y ** 2) + 0.01 * v[0:1],
             linear=lambda p: 1j * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: X.Int(np.abs(a) ** 2, [0, dx, 0], p),
                      lambda a, p: X.Int(np.real(a), [0, 0, dy], [[0, 0], [0, 0], [-1.5, 2.0]], p),
                      lambda a, p: X.Ave(a * np.conj(a), [0, 1, 0], p),
                      lambda a, p: np.abs(a) ** 2])
    o.pop("precision")
    return g, o


def test_partial_int_and_ave_match_oracle_block_means():
    from xspde_matlab_b200 import GpuPath, xpreferences
    g, o = _inputs()
    path = GpuPath(xpreferences([g])[0])
    shapes = path.av_shapes()
    assert shapes[0] == (1, 4, 1, 12) and shapes[1] == (1, 4, 16, 1) and shapes[2] == (1, 4, 1, 12)
    assert shapes[3] == (1, 4, 16, 12)
    for nc in (1, 2):
        av, _ = path.run_path(0, 2, nc)
        for b in range(2):
            ref, _ = oracle_block_av(o, b, nc)
            for k in range(4):
                e = rel_err(av[b][k].reshape(-1, order="F"), np.asarray(ref[k]).reshape(-1, order="F"))
                assert e < 1e-10, (nc, b, k, e)


def test_partial_int_through_xsim_matches_oracle_xsim():
    from xspde_matlab_b200 import xsim
    g, o = _inputs()
    eg, dg, _ = xsim(g)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        eo, do, _ = X.xsim(o)
    for a, b in zip(dg[0], do[0]):
        a, b = np.asarray(a), np.asarray(b)
        assert a.shape == b.shape
        assert np.allclose(a[..., 0], b[..., 0], rtol=1e-10, atol=1e-13)
