"""Block-granular checkpoint and resume of the host xsim (p.checkpoint): a run stopped after some
groups of blocks continues from the saved next block with the saved compensated moment sums and
returns exactly the moments of an uninterrupted run."""
import numpy as np
import pytest

from tests.test_dist_cpu import FakePath, _inputs


class StopAt(FakePath):
    """FakePath whose call for block `stop` fails, as a run killed there would stop."""

    def __init__(self, p, stop):
        super().__init__(p)
        self.stop = stop

    def run_path(self, first, nblocks, nc, a_in=None, a_out=False):
        if first <= self.stop < first + nblocks:
            raise RuntimeError("stopped at block %d" % self.stop)
        return super().run_path(first, nblocks, nc, a_in, a_out)


def _inp(tmp_path, blocks_per_save=2):
    inp = _inputs()
    inp[0].checkpoint = str(tmp_path / "run.npz")
    inp[0].checkpoint_blocks = blocks_per_save
    return inp


def test_resume_after_a_stop_equals_an_uninterrupted_run(tmp_path):
    from xspde_matlab_b200.xsim import _ensembles
    ref = _ensembles(_inputs(), [FakePath(_inputs()[0])])
    inp = _inp(tmp_path)
    with pytest.raises(RuntimeError, match="stopped at block 4"):
        _ensembles(inp, [StopAt(inp[0], 4)])
    z = np.load(tmp_path / "run.npz")
    assert int(z["next"]) == 4
    path = FakePath(inp[0])
    got = _ensembles(inp, [path])
    assert min(c[0] for c in path.calls) == 4  # blocks 0-3 were not integrated again
    for a, b in zip(got[0], ref[0]):
        assert np.array_equal(a, b)
    # a finished run's checkpoint returns its result without integrating anything
    path = FakePath(inp[0])
    again = _ensembles(inp, [path])
    assert not path.calls
    for a, b in zip(again[0], ref[0]):
        assert np.array_equal(a, b)


def test_checkpoint_of_another_run_is_refused(tmp_path):
    from xspde_matlab_b200.xsim import _ensembles
    inp = _inp(tmp_path)
    with pytest.raises(RuntimeError):
        _ensembles(inp, [StopAt(inp[0], 2)])
    other = _inp(tmp_path)
    other[0].seed = 99
    with pytest.raises(ValueError, match="different run"):
        _ensembles(other, [FakePath(other[0])])
