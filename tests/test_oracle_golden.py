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
