"""Helpers shared by the GPU parity tests: run one block through the oracle's
p.path (oracle/xspde_ref.py) and through the device path with the same inputs."""
import warnings

import numpy as np

from oracle import xspde_ref as X


def oracle_block_av(pdict, block, nc):
    """Block-mean observables av (list per observable) of the oracle's xpath for
    one ensemble block and check pass, with the Philox noise hooks."""
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        inp = X.xpreferences([pdict])
        p = inp[0].copy()
        p.block = block
        p.seq = 0
        p.dtr = p.dt / (2 * p.steps[0]) if (p.checks[0] and nc != 2) else p.dt / p.steps[0]
        p.propagator, p.da = p.propfactor(p)
        v = p.randomgen(p)
        p.t = p.origins[0]
        a = X.fit(np.asarray(X.call_cells(p.initial, None, v, p), dtype=complex), p.ca)
        X.initial_aux(a, nc, p)
        b, av, raw = p.path(a, nc, p)
    if p.rawdata:
        return av, b, raw
    return av, b


def rel_err(x, y):
    x = np.asarray(x)
    y = np.asarray(y)
    scale = max(np.max(np.abs(y)), 1e-300)
    return float(np.max(np.abs(x - y)) / scale)
