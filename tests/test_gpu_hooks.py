"""GPU replacements of the reference's per-call hooks against the oracle:
p.noisegen (xs_noise), p.randomgen (xs_random) and p.method (xs_step).
FP64: 1e-12 relative for the noise (same Philox words, libm vs CUDA math
rounding only) and 1e-10 for one method step."""
import numpy as np
import pytest

from oracle import xspde_ref as X
from tests.gpu_util import rel_err

pytestmark = pytest.mark.gpu

BASE = dict(dimensions=2, points=[5, 32], ranges=[0.4, 8.0], steps=2, ensembles=[6, 3, 1], noises=2, checks=1)


def _pair(method):
    g = dict(BASE, method=method, deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.3*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2 - 0.1", observe=["@(a,p) a"])
    o = dict(BASE, method=method,
             deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.3 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2 - 0.1, observe=[lambda a, p: a])
    from xspde_matlab_b200 import GpuPath, xpreferences
    return GpuPath(xpreferences([g])[0], path_kind=1), X.xpreferences([o])[0]


def test_noise_and_random_match_oracle():
    path, p = _pair("MP")
    for block in (0, 2):
        q = p.copy()
        q.block, q.seq, q.draw = block, 0, 7
        w_o = X.philox_noisegen(None, 1, p.nscale, q)
        w_g = path.noise(block, 7, p.nscale)
        assert rel_err(w_g, w_o) < 1e-12
        v_o = X.philox_randomgen(q)
        v_g = path.random(block)
        assert rel_err(v_g, v_o) < 1e-12


@pytest.mark.parametrize("method", ["MP", "RK4", "Euler", "RK2", "Implicit"])
def test_step_matches_oracle_method(method):
    path, p = _pair(method)
    rng = np.random.default_rng(3)
    a = (rng.standard_normal(p.ca) + 1j * rng.standard_normal(p.ca)) * 0.5
    w = rng.standard_normal([p.noises] + p.space + [p.ensembles[0]]) * 3.0
    q = p.copy()
    q.dtr = 0.05
    q.t = 0.3
    q.propagator, q.da = q.propfactor(q)
    ref = X.METHODS[method](a, w, q)
    got = path.step(a, w, 0.3, 0.05)
    assert rel_err(got, ref) < 1e-10
