"""GPU tests of the uneven batch (xs_batch_*): every item of a mixed batch,
integrated by one CUDA-graph launch, reproduces the single-problem p.path
replacement on the same input (same Philox noise, same kernels; only the
order of the FP64 observable sums differs: 1e-12 relative), one FP32 item
agrees with the CPU oracle (2e-4 relative, FP32 fields), autotuned tiles
leave the results unchanged, and relaunching the graph is deterministic."""
import numpy as np
import pytest

from tests.gpu_util import oracle_block_av, rel_err

pytestmark = pytest.mark.gpu

SUM_ORDER_TOL = 1e-12
FP32_TOL = 2e-4


def _items():
    from xspde_matlab_b200.batch import DRIFTS

    def item(drift, dim, N, g, steps, ntraj, seed, points=3):
        d = DRIFTS[drift]
        return dict(dimensions=dim + 1, fields=1, noises=1, inrandoms=1, points=[points] + [N] * dim,
                    ranges=[1.0] + [20.0] * dim, steps=steps, checks=0, ensembles=[ntraj, 1, 1], method="MP",
                    precision="fp32", seed=seed, g=g, deriv=d["deriv"], linear=d["linear%d" % dim],
                    initial=d["initial%d" % dim], observe=["@(a,p) abs(a).^2"])

    return [item("nls", 1, 32, 0.05, 10, 64, 1), item("nls", 1, 32, 0.01, 7, 128, 2),
            item("allen_cahn", 1, 256, 0.1, 5, 64, 3), item("nls", 2, 32, 0.03, 4, 64, 4),
            item("allen_cahn", 2, 64, 0.08, 3, 64, 5), item("nls", 2, 256, 0.02, 3, 64, 6),
            item("nls", 1, 1024, 0.005, 6, 192, 7), item("allen_cahn", 2, 128, 0.05, 3, 64, 8)]


def _single(inp):
    from xspde_matlab_b200 import GpuPath, xpreferences
    from xspde_matlab_b200.batch import _named_scalars
    p = xpreferences([_named_scalars(inp)])[0]
    av, _ = GpuPath(p, 0, runtime_params=True).run_path(0, 1, 1)
    return av[0]


def test_batch_items_match_single_problem_path():
    from xspde_matlab_b200.batch import Batch
    items = _items()
    b = Batch(items)
    s = b.summary()
    assert s["items"] == len(items) and s["streaming"] == 1 and s["variants"] == 6, s
    b.run()
    b.sync()
    for i, inp in enumerate(items):
        got = b.results(i)
        ref = _single(inp)
        for o in range(len(ref)):
            assert got[o].shape == ref[o].shape
            e = rel_err(got[o].reshape(-1), ref[o].reshape(-1))
            assert e < SUM_ORDER_TOL, (i, o, e, b.info(i))


def test_batch_item_matches_oracle():
    from xspde_matlab_b200.batch import Batch
    items = _items()[:2]
    b = Batch(items)
    b.run()
    b.sync()
    for i, inp in enumerate(items):
        g = inp["g"]
        o = {k: v for k, v in inp.items() if k not in ("deriv", "linear", "initial", "observe", "g", "precision")}
        o.update(deriv=lambda a, w, p, g=g: 1j * np.abs(a) ** 2 * a + 1j * g * a * w[0:1],
                 linear=lambda p: 0.5j * p.Dx ** 2, initial=lambda v, p: np.exp(-p.x ** 2 / 4) + 0 * v[0:1],
                 observe=[lambda a, p: np.abs(a) ** 2])
        av_o, _ = oracle_block_av(o, 0, 1)
        got = b.results(i)
        e = rel_err(got[0].reshape(-1, order="F"), av_o[0].reshape(-1, order="F"))
        assert e < FP32_TOL, (i, e)


def test_batch_autotune_and_relaunch_deterministic():
    from xspde_matlab_b200.batch import Batch
    items = _items()
    b0 = Batch(items)
    b0.run()
    b0.sync()
    ref = [b0.results(i) for i in range(len(items))]
    b = Batch(items)
    b.tune(1)
    tiles = [b.info(i) for i in range(len(items))]
    assert all(t["path"] == 2 or (t["G"] >= 1 and t["threads"] in (128, 256, 512, 1024)) for t in tiles), tiles
    b.run()
    b.sync()
    first = [b.results(i) for i in range(len(items))]
    b.run()
    b.run()
    b.sync()
    for i in range(len(items)):
        again = b.results(i)
        for o in range(len(ref[i])):
            assert np.array_equal(first[i][o], again[o]), (i, o)
            assert rel_err(first[i][o].reshape(-1), ref[i][o].reshape(-1)) < SUM_ORDER_TOL, (i, o, tiles[i])


def test_dpo_batch_fp64_matches_oracle():
    """Positive-P DPO (two coupled complex fields, multiplicative complex-sqrt
    noise, Stratonovich-corrected drift): each item has its own pump eps, read
    by the kernel as a runtime scalar; FP64 items agree with the oracle to 1e-10."""
    from xspde_matlab_b200.batch import Batch, dpo_instances
    items = [dict(d, ensembles=[256, 1, 1], points=[3], steps=10, ranges=[0.5])
             for d in dpo_instances(blocks=3, ntraj=256, precision="fp64")]
    b = Batch(items)
    assert b.summary()["variants"] == 1
    b.run()
    b.sync()
    for i, inp in enumerate(items):
        gam, eps, chi = (inp["params"][k] for k in ("gam", "eps", "chi"))

        def deriv(a, w, p, gam=gam, eps=eps, chi=chi):
            a1, a2 = a[0:1], a[1:2]
            return np.concatenate([
                -gam * a1 + eps * a2 - chi * a1 ** 2 * a2 + 0.5 * chi * a1 + np.sqrt(-chi * a1 ** 2 + 0j) * w[0:1],
                -gam * a2 + eps * a1 - chi * a2 ** 2 * a1 + 0.5 * chi * a2 + np.sqrt(-chi * a2 ** 2 + 0j) * w[1:2]])

        o = {k: v for k, v in inp.items() if k not in ("deriv", "initial", "observe", "params", "precision", "name")}
        o.update(deriv=deriv, initial=lambda v, p: np.array([[1.0 + 0j], [1.0 + 0j]]),
                 observe=[lambda a, p: np.real(a[0:1] * a[1:2]), lambda a, p: np.real(a[0:1])])
        av_o, _ = oracle_block_av(o, 0, 1)
        got = b.results(i)
        for k in range(2):
            e = rel_err(got[k].reshape(-1, order="F"), av_o[k].reshape(-1, order="F"))
            assert e < 1e-10, (i, k, e)


def test_batch_checked_items_run_both_passes():
    """Items with checks = 1 (Simulator/xensemble.m:41-45): the graph runs the
    fine pass (nc = 1) and the coarse pass (nc = 2, twice the step, mean of two
    fine draws) of every item, resident and streaming alike; each pass equals
    the single-problem path's pass on the same input (1e-12), and the FP64
    item's step error |fine - coarse| agrees with the oracle's to 1e-9
    relative (a difference of two close means)."""
    from xspde_matlab_b200.batch import Batch
    items = [dict(it, checks=1) for it in _items()[:6]]
    items[0] = dict(items[0], precision="fp64")
    b = Batch(items)
    s = b.summary()
    assert s["items"] == len(items) and s["streaming"] == 1, s
    b.run()
    b.sync()
    from xspde_matlab_b200 import GpuPath, xpreferences
    from xspde_matlab_b200.batch import _named_scalars
    for i, inp in enumerate(items):
        fine, coarse = b.passes(i)
        p = xpreferences([_named_scalars(inp)])[0]
        path = GpuPath(p, 0, runtime_params=True)
        for nc, got in ((1, fine), (2, coarse)):
            av, _ = path.run_path(0, 1, nc)
            ref = av[0]
            for o in range(len(ref)):
                e = rel_err(got[o].reshape(-1), ref[o].reshape(-1))
                assert e < SUM_ORDER_TOL, (i, nc, o, e, b.info(i))
        mean, err = b.results(i, step_error=True)
        assert np.array_equal(mean[0], fine[0]) and np.allclose(err[0], np.abs(fine[0] - coarse[0]))
    # the FP64 item against the oracle's two passes
    inp = items[0]
    g = inp["g"]
    o = {k: v for k, v in inp.items() if k not in ("deriv", "linear", "initial", "observe", "g", "precision")}
    o.update(deriv=lambda a, w, p, g=g: 1j * np.abs(a) ** 2 * a + 1j * g * a * w[0:1],
             linear=lambda p: 0.5j * p.Dx ** 2, initial=lambda v, p: np.exp(-p.x ** 2 / 4) + 0 * v[0:1],
             observe=[lambda a, p: np.abs(a) ** 2])
    f_o, _ = oracle_block_av(o, 0, 1)
    c_o, _ = oracle_block_av(o, 0, 2)
    fine, coarse = b.passes(0)
    assert rel_err(fine[0].reshape(-1, order="F"), f_o[0].reshape(-1, order="F")) < 1e-10
    assert rel_err(coarse[0].reshape(-1, order="F"), c_o[0].reshape(-1, order="F")) < 1e-10
    se = np.abs(fine[0] - coarse[0]).reshape(-1, order="F")
    se_o = np.abs(f_o[0] - c_o[0]).reshape(-1, order="F")
    assert np.max(se_o) > 0 and np.max(np.abs(se - se_o)) < 1e-9 * np.max(np.abs(f_o[0]))
